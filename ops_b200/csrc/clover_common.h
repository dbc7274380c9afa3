// Shared definitions of the CloverLeaf 2D hydro path: the constant block the
// loop kernels read and the field/state types the driver fills.
//
// state_type / grid_type / field_type keep the reference's member order
// (apps/c/CloverLeaf/user_types.h:25-52) because ops_decl_const copies them
// as raw bytes; FIELD_* indices follow user_types.h:4-19.
#pragma once

namespace opsb {
namespace clover {

enum {
  FIELD_DENSITY0 = 0, FIELD_DENSITY1, FIELD_ENERGY0, FIELD_ENERGY1, FIELD_PRESSURE, FIELD_VISCOSITY,
  FIELD_SOUNDSPEED, FIELD_XVEL0, FIELD_XVEL1, FIELD_YVEL0, FIELD_YVEL1, FIELD_VOL_FLUX_X, FIELD_VOL_FLUX_Y,
  FIELD_MASS_FLUX_X, FIELD_MASS_FLUX_Y, NUM_FIELDS
};

enum { G_RECT = 1, G_CIRC = 2, G_POINT = 3 };
constexpr int kMaxStates = 24;

struct state_type {
  int defined;
  double density, energy, xvel, yvel;
  int geometry;
  double xmin, xmax, ymin, ymax, radius;
};

struct grid_type {
  double xmin, ymin, xmax, ymax;
  int x_cells, y_cells;
};

struct field_type {
  int left, right, bottom, top, left_boundary, right_boundary, bottom_boundary, top_boundary;
  int x_min, y_min, x_max, y_max;
};

// Everything the loop kernels read besides their arguments
// (the ops_decl_const list of apps/c/CloverLeaf/clover_leaf.cpp:147-160).
struct Consts {
  double g_small, g_big;
  double dtc_safe, dtu_safe, dtv_safe, dtdiv_safe;
  double dt;
  field_type field;
  grid_type grid;
  int number_of_states;
  int g_circ, g_point, g_rect;
  state_type states[kMaxStates];
};

}  // namespace clover
}  // namespace opsb
