// Shared definitions of the CloverLeaf 3D hydro path: the constant block the
// loop kernels read and the field/state types the driver fills.
//
// state_type / grid_type / field_type keep the reference's member order
// (apps/c/CloverLeaf_3D/user_types.h:24-55) because ops_decl_const copies
// them as raw bytes; FIELD_* indices follow user_types.h:4-23.
#pragma once

namespace opsb {
namespace clover3d {

enum {
  FIELD_DENSITY0 = 0, FIELD_DENSITY1, FIELD_ENERGY0, FIELD_ENERGY1, FIELD_PRESSURE, FIELD_VISCOSITY,
  FIELD_SOUNDSPEED, FIELD_XVEL0, FIELD_XVEL1, FIELD_YVEL0, FIELD_YVEL1, FIELD_ZVEL0, FIELD_ZVEL1,
  FIELD_VOL_FLUX_X, FIELD_VOL_FLUX_Y, FIELD_VOL_FLUX_Z, FIELD_MASS_FLUX_X, FIELD_MASS_FLUX_Y, FIELD_MASS_FLUX_Z,
  NUM_FIELDS
};

enum { G_CUBE = 1, G_SPHE = 2, G_POINT = 3 };
enum { G_XDIR = 1, G_YDIR = 2, G_ZDIR = 3 };
constexpr int kMaxStates = 16;

struct state_type {
  int defined;
  double density, energy, xvel, yvel, zvel;
  int geometry;
  double xmin, xmax, ymin, ymax, zmin, zmax, radius;
};

struct grid_type {
  double xmin, ymin, xmax, ymax, zmin, zmax;
  int x_cells, y_cells, z_cells;
};

struct field_type {
  int left, right, bottom, top, back, front, left_boundary, right_boundary, bottom_boundary, top_boundary,
      back_boundary, front_boundary;
  int x_min, y_min, x_max, y_max, z_min, z_max;
};

// Everything the loop kernels read besides their arguments
// (the ops_decl_const list of apps/c/CloverLeaf_3D/clover_leaf.cpp:150-169).
struct Consts {
  double g_small, g_big;
  double dtc_safe, dtu_safe, dtv_safe, dtw_safe, dtdiv_safe;
  double dt;
  field_type field;
  grid_type grid;
  int number_of_states;
  int g_sphe, g_point, g_cube;
  state_type states[kMaxStates];
};

}  // namespace clover3d
}  // namespace opsb
