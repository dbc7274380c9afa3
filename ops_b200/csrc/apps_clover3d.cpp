// CloverLeaf 3D driver on the OPS-B200 runtime: the loop sequence of the
// reference app (apps/c/CloverLeaf_3D/clover_leaf.cpp:133-213 and the files
// it calls, cited per function), with the input deck passed as a struct
// instead of clover.in. Every ops_par_loop keeps the reference's kernel,
// range, stencils and access modes, including the places where the
// reference's choices look accidental (argument flags in update_halo,
// zvel0(1,0,0) read twice in flux_calc_kernelz, a geometry flag that is not
// reset between states): results follow the reference, not an idealised
// scheme.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/ops_b200.h"
#include "clover3d_common.h"
#include "runtime.h"

namespace opsb {
int capi_guard(const std::function<int()> &f);

namespace clover3d {

struct Clover3D {
  Runtime &r;
  // run-time constants and state (clover_leaf.cpp:73-131, read_input.cpp:44-80)
  double g_small = 1.0e-16, g_big = 1.0e+21;
  double dtold = 0, dt = 0, clover_time = 0, dtinit = 0.1, dtmin = 0.0000001, dtmax = 1.0, dtrise = 1.05;
  double dtc_safe = 0.75, dtu_safe = 0.5, dtv_safe = 0.5, dtw_safe = 0.5, dtdiv_safe = 0.5;
  double end_time = 10.0;
  int end_step = 640000, summary_frequency = 10;
  int step = 0, advect_x = 1, complete = 0;
  int g_cube = G_CUBE, g_sphe = G_SPHE, g_point = G_POINT;
  int number_of_states = 0;
  state_type states[kMaxStates];
  grid_type grid;
  field_type field;
  int fields[NUM_FIELDS] = {0};  // persists between calls, as the reference's global does
  int jdt = 0, kdt = 0;

  int clover_grid = -1;
  int density0, density1, energy0, energy1, pressure, viscosity, soundspeed, volume;
  int xvel0, xvel1, yvel0, yvel1, zvel0, zvel1;
  int vol_flux_x, vol_flux_y, vol_flux_z, mass_flux_x, mass_flux_y, mass_flux_z, xarea, yarea, zarea;
  int work_array1, work_array2, work_array3, work_array4, work_array5, work_array6, work_array7;
  int cellx, celly, cellz, vertexx, vertexy, vertexz, celldx, celldy, celldz, vertexdx, vertexdy, vertexdz;
  int xx, yy, zz;

  int S000, S_P100, S_0P10, S_00P1, S_M100, S_0M10, S_00M1;
  int S_f0M1M1, S_fM10M1, S_fM1M10, S_f0P1P1, S_fP10P1, S_fP1P10;
  int S_fP1P1P1, S_fP1M1M1, S_fM1P1M1, S_fM1M1P1, S_fM1P1P1, S_fP1M1P1, S_fP1P1M1, S_fM1M1M1;
  int S_P200, S_0P20, S_00P2, S_M200, S_0M20, S_00M2, S_P300, S_0P30, S_00P3, S_M300, S_0M30, S_00M3;
  int S_P400, S_0P40, S_00P4, S_M400, S_0M40, S_00M4;
  int S_P100_P200_M100, S_0P10_0P20_0M10, S_00P1_00P2_00M1;
  int S_P100_M100_M200, S_0P10_0M10_0M20, S_00P1_00M1_00M2, S_6PT;
  int S_STRID_X, S_STRID_Y, S_STRID_Z, S_P100_STRID_X, S_0P10_STRID_Y, S_00P1_STRID_Z;
  int S_P100_M100_STRID_X, S_0P10_0M10_STRID_Y, S_00P1_00M1_STRID_Z;
  int S_P100_M100_M200_STRID_X, S_0P10_0M10_0M20_STRID_Y, S_00P1_00M1_00M2_STRID_Z;
  int red_local_dt, red_xl_pos, red_yl_pos, red_zl_pos, red_vol, red_mass, red_ie, red_ke, red_press, red_output;

  std::vector<double> summaries;  // per field_summary: step, time, vol, mass, ie, ke, press, dt
  long long halo_loops_skipped = 0;

  explicit Clover3D(Runtime &rt) : r(rt) {
    memset(states, 0, sizeof(states));
    memset(&grid, 0, sizeof(grid));
    memset(&field, 0, sizeof(field));
  }

  PrefixedLoops loops{"cloverleaf3d/"};
  void loop(const char *k, const char *name, const int *range, std::initializer_list<Arg> a) {
    r.par_loop(loops.get(k), name, clover_grid, 3, range, a.begin(), (int)a.size());
  }
  void loop(const char *k, const int *range, std::initializer_list<Arg> a) { loop(k, k, range, a); }
  Arg dat(int d, int s, int acc) { return arg_dat(d, 1, s, acc); }
  Arg dat_opt(int d, int s, int acc, int flag) { return arg_dat_opt(d, 1, s, acc, flag); }
  void set_fields(std::initializer_list<int> on) {
    for (int i = 0; i < NUM_FIELDS; i++) fields[i] = 0;
    for (int i : on) fields[i] = 1;
  }

  // read_input.cpp:37-276 (deck values already parsed by the caller).
  void read_input(const ops_b200_clover3d_deck &d) {
    grid.xmin = d.xmin; grid.ymin = d.ymin; grid.zmin = d.zmin;
    grid.xmax = d.xmax; grid.ymax = d.ymax; grid.zmax = d.zmax;
    grid.x_cells = d.x_cells; grid.y_cells = d.y_cells; grid.z_cells = d.z_cells;
    dtinit = d.initial_timestep; dtmax = d.max_timestep; dtrise = d.timestep_rise;
    end_time = d.end_time; end_step = d.end_step; summary_frequency = d.summary_frequency;
    number_of_states = d.number_of_states;
    if (number_of_states < 1 || number_of_states > kMaxStates) throw Error(E_ARG, "1..16 states are supported");
    for (int i = 0; i < number_of_states; i++) {
      const ops_b200_clover3d_state &s = d.states[i];
      states[i].defined = 1;
      states[i].density = s.density; states[i].energy = s.energy;
      states[i].xvel = s.xvel; states[i].yvel = s.yvel; states[i].zvel = s.zvel;
      states[i].geometry = s.geometry;
      states[i].xmin = s.xmin; states[i].xmax = s.xmax; states[i].ymin = s.ymin; states[i].ymax = s.ymax;
      states[i].zmin = s.zmin; states[i].zmax = s.zmax; states[i].radius = s.radius;
    }
    field.x_min = 0 + 2; field.y_min = 0 + 2; field.z_min = 0 + 2;
    field.x_max = grid.x_cells + 2; field.y_max = grid.y_cells + 2; field.z_max = grid.z_cells + 2;
    field.left = 0; field.bottom = 0; field.back = 0;
    // read_input.cpp:262-275: the state boxes shrink by 1 % of a cell, with
    // the cell width rounded to single precision as the reference does.
    float dx = (grid.xmax - grid.xmin) / (float)(grid.x_cells);
    float dy = (grid.ymax - grid.ymin) / (float)(grid.y_cells);
    float dz = (grid.zmax - grid.zmin) / (float)(grid.z_cells);
    for (int i = 0; i < number_of_states; i++) {
      states[i].xmin = states[i].xmin + (dx / 100.00);
      states[i].ymin = states[i].ymin + (dy / 100.00);
      states[i].zmin = states[i].zmin + (dz / 100.00);
      states[i].xmax = states[i].xmax - (dx / 100.00);
      states[i].ymax = states[i].ymax - (dy / 100.00);
      states[i].zmax = states[i].zmax - (dz / 100.00);
    }
  }

  int stencil(int points, std::initializer_list<int> offs, const char *name) {
    std::vector<int> o(offs);
    return r.decl_stencil(3, points, o.data(), nullptr, name);
  }
  int strided(int points, std::initializer_list<int> offs, std::initializer_list<int> stride, const char *name) {
    std::vector<int> o(offs), s(stride);
    return r.decl_stencil(3, points, o.data(), s.data(), name);
  }

  // build_field.cpp:35-297
  void build_field() {
    const int xc = grid.x_cells, yc = grid.y_cells, zc = grid.z_cells;
    clover_grid = r.decl_block(3, "clover grid");
    int d_p[3] = {2, 2, 2}, d_m[3] = {-2, -2, -2}, base[3] = {0, 0, 0};
    int size[3] = {xc + 5, yc + 5, zc + 5};
    auto D = [&](const char *n) { return r.decl_dat(clover_grid, 1, size, base, d_m, d_p, nullptr, 8, "double", n); };
    density0 = D("density0"); density1 = D("density1"); energy0 = D("energy0"); energy1 = D("energy1");
    pressure = D("pressure"); viscosity = D("viscosity"); soundspeed = D("soundspeed"); volume = D("volume");
    size[0]++; size[1]++; size[2]++;
    xvel0 = D("xvel0"); xvel1 = D("xvel1"); yvel0 = D("yvel0"); yvel1 = D("yvel1");
    zvel0 = D("zvel0"); zvel1 = D("zvel1");
    work_array1 = D("work_array1"); work_array2 = D("work_array2"); work_array3 = D("work_array3");
    work_array4 = D("work_array4"); work_array5 = D("work_array5"); work_array6 = D("work_array6");
    work_array7 = D("work_array7");
    size[0] = xc + 5; size[1] = yc + 5; size[2] = zc + 5;
    vol_flux_x = D("vol_flux_x"); mass_flux_x = D("mass_flux_x"); xarea = D("xarea");
    vol_flux_y = D("vol_flux_y"); mass_flux_y = D("mass_flux_y"); yarea = D("yarea");
    vol_flux_z = D("vol_flux_z"); mass_flux_z = D("mass_flux_z"); zarea = D("zarea");
    // one-dimensional coordinate dats (build_field.cpp:105-146)
    auto D1 = [&](int axis, int n, const char *type, const char *nm) {
      int sz[3] = {1, 1, 1}, dm[3] = {0, 0, 0}, dp[3] = {0, 0, 0};
      sz[axis] = n; dm[axis] = -2; dp[axis] = 2;
      return r.decl_dat(clover_grid, 1, sz, base, dm, dp, nullptr, 0, type, nm);
    };
    cellx = D1(0, xc + 5, "double", "cellx"); celldx = D1(0, xc + 5, "double", "celldx");
    celly = D1(1, yc + 5, "double", "celly"); celldy = D1(1, yc + 5, "double", "celldy");
    cellz = D1(2, zc + 5, "double", "cellz"); celldz = D1(2, zc + 5, "double", "celldz");
    vertexx = D1(0, xc + 6, "double", "vertexx"); vertexdx = D1(0, xc + 6, "double", "vertexdx");
    vertexy = D1(1, yc + 6, "double", "vertexy"); vertexdy = D1(1, yc + 6, "double", "vertexdy");
    vertexz = D1(2, zc + 6, "double", "vertexz"); vertexdz = D1(2, zc + 6, "double", "vertexdz");
    xx = D1(0, xc + 6, "int", "xx"); yy = D1(1, yc + 6, "int", "yy"); zz = D1(2, zc + 6, "int", "zz");

    S000 = stencil(1, {0, 0, 0}, "0,0,0");
    S_P100 = stencil(2, {0, 0, 0, 1, 0, 0}, "0,0,0:1,0,0");
    S_0P10 = stencil(2, {0, 0, 0, 0, 1, 0}, "0,0,0:0,1,0");
    S_00P1 = stencil(2, {0, 0, 0, 0, 0, 1}, "0,0,0:0,0,1");
    S_M100 = stencil(2, {0, 0, 0, -1, 0, 0}, "0,0,0:-1,0,0");
    S_0M10 = stencil(2, {0, 0, 0, 0, -1, 0}, "0,0,0:0,-1,0");
    S_00M1 = stencil(2, {0, 0, 0, 0, 0, -1}, "0,0,0:0,0,-1");
    S_f0M1M1 = stencil(4, {0, 0, 0, 0, -1, 0, 0, 0, -1, 0, -1, -1}, "f0,0,0:0,-1,-1");
    S_fM10M1 = stencil(4, {0, 0, 0, -1, 0, 0, 0, 0, -1, -1, 0, -1}, "f0,0,0:-1,0,-1");
    S_fM1M10 = stencil(4, {0, 0, 0, 0, -1, 0, -1, 0, 0, -1, -1, 0}, "f0,0,0:-1,-1,0");
    S_f0P1P1 = stencil(4, {0, 0, 0, 0, 1, 0, 0, 0, 1, 0, 1, 1}, "f0,0,0:0,1,1");
    S_fP10P1 = stencil(4, {0, 0, 0, 1, 0, 0, 0, 0, 1, 1, 0, 1}, "f0,0,0:1,0,1");
    S_fP1P10 = stencil(4, {0, 0, 0, 0, 1, 0, 1, 0, 0, 1, 1, 0}, "f0,0,0:1,1,0");
    S_fP1P1P1 = stencil(8, {0, 0, 0, 1, 0, 0, 1, 1, 0, 1, 1, 1, 0, 1, 0, 0, 1, 1, 0, 0, 1, 1, 0, 1}, "f0,0,0:1,1,1");
    S_fP1M1M1 = stencil(8, {0, 0, 0, 1, 0, 0, 1, -1, 0, 1, -1, -1, 0, -1, 0, 0, -1, -1, 0, 0, -1, 1, 0, -1},
                        "f0,0,0:1,-1,-1");
    S_fM1P1M1 = stencil(8, {0, 0, 0, -1, 0, 0, -1, 1, 0, -1, 1, -1, 0, 1, 0, 0, 1, -1, 0, 0, -1, -1, 0, -1},
                        "f0,0,0:-1,1,-1");
    S_fM1M1P1 = stencil(8, {0, 0, 0, -1, 0, 0, -1, -1, 0, -1, -1, 1, 0, -1, 0, 0, -1, 1, 0, 0, 1, -1, 0, 1},
                        "f0,0,0:-1,-1,1");
    S_fM1P1P1 = stencil(8, {0, 0, 0, -1, 0, 0, -1, 1, 0, -1, 1, 1, 0, 1, 0, 0, 1, 1, 0, 0, 1, -1, 0, 1},
                        "f0,0,0:-1,1,1");
    S_fP1M1P1 = stencil(8, {0, 0, 0, 1, 0, 0, 1, -1, 0, 1, -1, 1, 0, -1, 0, 0, -1, 1, 0, 0, 1, 1, 0, 1},
                        "f0,0,0:1,-1,1");
    S_fP1P1M1 = stencil(8, {0, 0, 0, 1, 0, 0, 1, 1, 0, 1, 1, -1, 0, 1, 0, 0, 1, -1, 0, 0, -1, 1, 0, -1},
                        "f0,0,0:1,1,-1");
    S_fM1M1M1 = stencil(8, {0, 0, 0, -1, 0, 0, -1, -1, 0, -1, -1, -1, 0, -1, 0, 0, -1, -1, 0, 0, -1, -1, 0, -1},
                        "f0,0,0:-1,-1,-1");
    S_P200 = stencil(2, {0, 0, 0, 2, 0, 0}, "0,0,0:2,0,0");
    S_0P20 = stencil(2, {0, 0, 0, 0, 2, 0}, "0,0,0:0,2,0");
    S_00P2 = stencil(2, {0, 0, 0, 0, 0, 2}, "0,0,0:0,0,2");
    S_M200 = stencil(2, {0, 0, 0, -2, 0, 0}, "0,0,0:-2,0,0");
    S_0M20 = stencil(2, {0, 0, 0, 0, -2, 0}, "0,0,0:0,-2,0");
    S_00M2 = stencil(2, {0, 0, 0, 0, 0, -2}, "0,0,0:0,0,-2");
    S_P300 = stencil(2, {0, 0, 0, 3, 0, 0}, "0,0,0:3,0,0");
    S_0P30 = stencil(2, {0, 0, 0, 0, 3, 0}, "0,0,0:0,3,0");
    S_00P3 = stencil(2, {0, 0, 0, 0, 0, 3}, "0,0,0:0,0,3");
    S_M300 = stencil(2, {0, 0, 0, -3, 0, 0}, "0,0,0:-3,0,0");
    S_0M30 = stencil(2, {0, 0, 0, 0, -3, 0}, "0,0,0:0,-3,0");
    S_00M3 = stencil(2, {0, 0, 0, 0, 0, -3}, "0,0,0:0,0,-3");
    S_P400 = stencil(2, {0, 0, 0, 4, 0, 0}, "0,0,0:4,0,0");
    S_0P40 = stencil(2, {0, 0, 0, 0, 4, 0}, "0,0,0:0,4,0");
    S_00P4 = stencil(2, {0, 0, 0, 0, 0, 4}, "0,0,0:0,0,4");
    S_M400 = stencil(2, {0, 0, 0, -4, 0, 0}, "0,0,0:-4,0,0");
    S_0M40 = stencil(2, {0, 0, 0, 0, -4, 0}, "0,0,0:0,-4,0");
    S_00M4 = stencil(2, {0, 0, 0, 0, 0, -4}, "0,0,0:0,0,-4");
    S_P100_P200_M100 = stencil(4, {0, 0, 0, 1, 0, 0, 2, 0, 0, -1, 0, 0}, "0,0,0:1,0,0:2,0,0:-1,0,0");
    S_0P10_0P20_0M10 = stencil(4, {0, 0, 0, 0, 1, 0, 0, 2, 0, 0, -1, 0}, "0,0,0:0,1,0:0,2,0:0,-1,0");
    S_00P1_00P2_00M1 = stencil(4, {0, 0, 0, 0, 0, 1, 0, 0, 2, 0, 0, -1}, "0,0,0:0,0,1:0,0,2:0,0,-1");
    S_P100_M100_M200 = stencil(4, {0, 0, 0, 1, 0, 0, -1, 0, 0, -2, 0, 0}, "0,0,0:1,0,0:-1,0,0:-2,0,0");
    S_0P10_0M10_0M20 = stencil(4, {0, 0, 0, 0, 1, 0, 0, -1, 0, 0, -2, 0}, "0,0,0:0,1,0:0,-1,0:0,-2,0");
    S_00P1_00M1_00M2 = stencil(4, {0, 0, 0, 0, 0, 1, 0, 0, -1, 0, 0, -2}, "0,0,0:0,0,1:0,0,-1:0,0,-2");
    S_6PT = stencil(6, {1, 0, 0, -1, 0, 0, 0, 1, 0, 0, -1, 0, 0, 0, 1, 0, 0, -1}, "6pt");
    S_STRID_X = strided(1, {0, 0, 0}, {1, 0, 0}, "s3D_000_stride3D_x");
    S_STRID_Y = strided(1, {0, 0, 0}, {0, 1, 0}, "s3D_000_stride3D_y");
    S_STRID_Z = strided(1, {0, 0, 0}, {0, 0, 1}, "s3D_000_stride3D_z");
    S_P100_STRID_X = strided(2, {0, 0, 0, 1, 0, 0}, {1, 0, 0}, "s3D_000_P100_stride3D_x");
    S_0P10_STRID_Y = strided(2, {0, 0, 0, 0, 1, 0}, {0, 1, 0}, "s3D_000_0P10_stride3D_y");
    S_00P1_STRID_Z = strided(2, {0, 0, 0, 0, 0, 1}, {0, 0, 1}, "s3D_000_00P1_stride3D_z");
    S_P100_M100_STRID_X = strided(3, {0, 0, 0, 1, 0, 0, -1, 0, 0}, {1, 0, 0}, "s3D_000_P100_M100_stride3D_x");
    S_0P10_0M10_STRID_Y = strided(3, {0, 0, 0, 0, 1, 0, 0, -1, 0}, {0, 1, 0}, "s3D_000_0P10_0M10_stride3D_y");
    S_00P1_00M1_STRID_Z = strided(3, {0, 0, 0, 0, 0, 1, 0, 0, -1}, {0, 0, 1}, "s3D_000_00P1_00M1_stride3D_z");
    // the reference declares these three with the +1,+2,-1 point lists
    // (build_field.cpp:211-213), whatever their names say
    S_P100_M100_M200_STRID_X = strided(4, {0, 0, 0, 1, 0, 0, 2, 0, 0, -1, 0, 0}, {1, 0, 0}, "x4");
    S_0P10_0M10_0M20_STRID_Y = strided(4, {0, 0, 0, 0, 1, 0, 0, 2, 0, 0, -1, 0}, {0, 1, 0}, "y4");
    S_00P1_00M1_00M2_STRID_Z = strided(4, {0, 0, 0, 0, 0, 1, 0, 0, 2, 0, 0, -1}, {0, 0, 1}, "z4");

    red_local_dt = r.decl_reduction(8, "double", "local_dt");
    red_xl_pos = r.decl_reduction(8, "double", "xl_pos");
    red_yl_pos = r.decl_reduction(8, "double", "yl_pos");
    red_zl_pos = r.decl_reduction(8, "double", "zl_pos");
    red_vol = r.decl_reduction(8, "double", "vol");
    red_mass = r.decl_reduction(8, "double", "mass");
    red_ie = r.decl_reduction(8, "double", "ie");
    red_ke = r.decl_reduction(8, "double", "ke");
    red_press = r.decl_reduction(8, "double", "press");
    red_output = r.decl_reduction(28 * 8, "double", "output");
  }

  // initialise_chunk.cpp:37-121
  void initialise_chunk() {
    const int x_min = field.x_min, x_max = field.x_max, y_min = field.y_min, y_max = field.y_max;
    const int z_min = field.z_min, z_max = field.z_max;
    int rangex[] = {x_min - 2, x_max + 3, y_min - 2, y_max + 3, z_min - 2, z_max + 3};
    int rangey[] = {x_min - 2, x_max + 3, y_min - 2, y_max + 3, z_min - 2, z_max + 3};
    int rangez[] = {x_min - 2, x_max + 3, y_min - 2, y_max + 3, z_min - 2, z_max + 3};
    int rangefull[] = {-2, grid.x_cells + 8, -2, grid.y_cells + 8, -2, grid.z_cells + 8};
    loop("initialise_chunk_kernel_xx", rangefull, {dat(xx, S_STRID_X, ACC_WRITE), arg_idx()});
    loop("initialise_chunk_kernel_yy", rangefull, {dat(yy, S_STRID_Y, ACC_WRITE), arg_idx()});
    loop("initialise_chunk_kernel_zz", rangefull, {dat(zz, S_STRID_Z, ACC_WRITE), arg_idx()});
    loop("initialise_chunk_kernel_x", rangex,
         {dat(vertexx, S_STRID_X, ACC_WRITE), dat(xx, S_STRID_X, ACC_READ), dat(vertexdx, S_STRID_X, ACC_WRITE)});
    loop("initialise_chunk_kernel_y", rangey,
         {dat(vertexy, S_STRID_Y, ACC_WRITE), dat(yy, S_STRID_Y, ACC_READ), dat(vertexdy, S_STRID_Y, ACC_WRITE)});
    loop("initialise_chunk_kernel_z", rangez,
         {dat(vertexz, S_STRID_Z, ACC_WRITE), dat(zz, S_STRID_Z, ACC_READ), dat(vertexdz, S_STRID_Z, ACC_WRITE)});
    rangex[0] = x_min - 2; rangex[1] = x_max + 2;
    loop("initialise_chunk_kernel_cellx", rangex,
         {dat(vertexx, S_P100_STRID_X, ACC_READ), dat(cellx, S_STRID_X, ACC_WRITE), dat(celldx, S_STRID_X, ACC_WRITE)});
    rangey[2] = y_min - 2; rangey[3] = y_max + 2;
    loop("initialise_chunk_kernel_celly", rangey,
         {dat(vertexy, S_0P10_STRID_Y, ACC_READ), dat(celly, S_STRID_Y, ACC_WRITE), dat(celldy, S_STRID_Y, ACC_WRITE)});
    rangez[4] = z_min - 2; rangez[5] = z_max + 2;
    loop("initialise_chunk_kernel_cellz", rangez,
         {dat(vertexz, S_00P1_STRID_Z, ACC_READ), dat(cellz, S_STRID_Z, ACC_WRITE), dat(celldz, S_STRID_Z, ACC_WRITE)});
    int rangexyz[] = {x_min - 2, x_max + 2, y_min - 2, y_max + 2, z_min - 2, z_max + 2};
    loop("initialise_chunk_kernel_volume", rangexyz,
         {dat(volume, S000, ACC_WRITE), dat(celldy, S_STRID_Y, ACC_READ), dat(xarea, S000, ACC_WRITE),
          dat(celldx, S_STRID_X, ACC_READ), dat(yarea, S000, ACC_WRITE), dat(celldz, S_STRID_Z, ACC_READ),
          dat(zarea, S000, ACC_WRITE)});
  }

  void generate() {  // generate.cpp:37-66
    int rangexyz[] = {field.x_min - 2, field.x_max + 2, field.y_min - 2, field.y_max + 2, field.z_min - 2,
                      field.z_max + 2};
    loop("generate_chunk_kernel", rangexyz,
         {dat(vertexx, S_P100_M100_STRID_X, ACC_READ), dat(vertexy, S_0P10_0M10_STRID_Y, ACC_READ),
          dat(vertexz, S_00P1_00M1_STRID_Z, ACC_READ), dat(energy0, S000, ACC_WRITE), dat(density0, S000, ACC_WRITE),
          dat(xvel0, S000, ACC_WRITE), dat(yvel0, S000, ACC_WRITE), dat(zvel0, S000, ACC_WRITE),
          dat(cellx, S_P100_M100_STRID_X, ACC_READ), dat(celly, S_0P10_0M10_STRID_Y, ACC_READ),
          dat(cellz, S_00P1_00M1_STRID_Z, ACC_READ)});
  }

  const int *inner(int *rng, int px = 0, int py = 0, int pz = 0) {
    rng[0] = field.x_min; rng[1] = field.x_max + px;
    rng[2] = field.y_min; rng[3] = field.y_max + py;
    rng[4] = field.z_min; rng[5] = field.z_max + pz;
    return rng;
  }

  void ideal_gas(int predict) {  // ideal_gas.cpp:38-68
    int rng[6];
    int d = predict ? density1 : density0, e = predict ? energy1 : energy0;
    loop("ideal_gas_kernel", inner(rng),
         {dat(d, S000, ACC_READ), dat(e, S000, ACC_READ), dat(pressure, S000, ACC_WRITE),
          dat(soundspeed, S000, ACC_WRITE)});
  }

  // update_halo.cpp:41-665: every face loop runs unconditionally in the
  // reference and its kernel tests the field flags itself. A loop whose
  // kernel would test only clear flags writes nothing and is not queued
  // (counted in halo_loops_skipped); the flags it is queued with are the
  // reference's, including the crossed ones of update_halo_kernel1_fr1.
  void update_halo(const int *f, int depth) {
    const int x_min = field.x_min, x_max = field.x_max, y_min = field.y_min, y_max = field.y_max;
    const int z_min = field.z_min, z_max = field.z_max, d = depth;
    Arg gbl = arg_gbl(f, NUM_FIELDS, 4, ACC_READ);
    auto R = [](int a, int b, int c, int e, int g, int h) { return std::vector<int>{a, b, c, e, g, h}; };
    // cell-centred fields
    const bool any1 = f[FIELD_DENSITY0] || f[FIELD_DENSITY1] || f[FIELD_ENERGY0] || f[FIELD_ENERGY1] ||
                      f[FIELD_PRESSURE] || f[FIELD_VISCOSITY] || f[FIELD_SOUNDSPEED];
    auto k1 = [&](const char *k, const char *nm, std::vector<int> rng, int st, bool crossed = false) {
      if (!any1) {
        halo_loops_skipped++;
        return;
      }
      loop(k, nm, rng.data(),
           {dat_opt(density0, st, ACC_RW, f[FIELD_DENSITY0]), dat_opt(density1, st, ACC_RW, f[FIELD_DENSITY1]),
            dat_opt(energy0, st, ACC_RW, f[crossed ? FIELD_ENERGY1 : FIELD_ENERGY0]),
            dat_opt(energy1, st, ACC_RW, f[crossed ? FIELD_DENSITY0 : FIELD_ENERGY1]),
            dat_opt(pressure, st, ACC_RW, f[FIELD_PRESSURE]), dat_opt(viscosity, st, ACC_RW, f[FIELD_VISCOSITY]),
            dat_opt(soundspeed, st, ACC_RW, f[FIELD_SOUNDSPEED]), gbl});
    };
    if (d == 2) k1("update_halo_kernel1_b2", "update_halo_kernel1", R(x_min - d, x_max + d, y_min - 2, y_min - 1, z_min - d, z_max + d), S_0P30);
    k1("update_halo_kernel1_b1", "update_halo_kernel1", R(x_min - d, x_max + d, y_min - 1, y_min, z_min - d, z_max + d), S_0P10);
    if (d == 2) k1("update_halo_kernel1_t2", "update_halo_kernel1", R(x_min - d, x_max + d, y_max + 1, y_max + 2, z_min - d, z_max + d), S_0M30);
    k1("update_halo_kernel1_t1", "update_halo_kernel1", R(x_min - d, x_max + d, y_max, y_max + 1, z_min - d, z_max + d), S_0M10);
    if (d == 2) k1("update_halo_kernel1_l2", "update_halo_kernel", R(x_min - 2, x_min - 1, y_min - d, y_max + d, z_min - d, z_max + d), S_P300);
    k1("update_halo_kernel1_l1", "update_halo_kernel", R(x_min - 1, x_min, y_min - d, y_max + d, z_min - d, z_max + d), S_P100);
    if (d == 2) k1("update_halo_kernel1_r2", "update_halo_kernel", R(x_max + 1, x_max + 2, y_min - d, y_max + d, z_min - d, z_max + d), S_M300);
    k1("update_halo_kernel1_r1", "update_halo_kernel", R(x_max, x_max + 1, y_min - d, y_max + d, z_min - d, z_max + d), S_M100);
    if (d == 2) k1("update_halo_kernel1_ba2", "update_halo_kernel", R(x_min - d, x_max + d, y_min - d, y_max + d, z_min - 2, z_min - 1), S_00P3);
    k1("update_halo_kernel1_ba1", "update_halo_kernel", R(x_min - d, x_max + d, y_min - d, y_max + d, z_min - 1, z_min), S_00P1);
    if (d == 2) k1("update_halo_kernel1_fr2", "update_halo_kernel", R(x_min - d, x_max + d, y_min - d, y_max + d, z_max + 1, z_max + 2), S_00M3);
    k1("update_halo_kernel1_fr1", "update_halo_kernel", R(x_min - d, x_max + d, y_min - d, y_max + d, z_max, z_max + 1), S_00M1, true);

    // pairs of node or face fields
    auto k2 = [&](const char *k, std::vector<int> rng, int a, int fa, int b, int fb, int st) {
      if (!f[fa] && !f[fb]) {
        halo_loops_skipped++;
        return;
      }
      loop(k, rng.data(), {dat_opt(a, st, ACC_RW, f[fa]), dat_opt(b, st, ACC_RW, f[fb]), gbl});
    };
    // velocities: the same twelve ranges for x, y and z (rangexy_*b)
    struct Vel { int a, fa, b, fb; const char *names[12]; };
    const Vel vels[3] = {
        {xvel0, FIELD_XVEL0, xvel1, FIELD_XVEL1,
         {"update_halo_kernel2_xvel_plus_4_bot", "update_halo_kernel2_xvel_plus_2_bot",
          "update_halo_kernel2_xvel_plus_4_top", "update_halo_kernel2_xvel_plus_2_top",
          "update_halo_kernel2_xvel_minus_4_left", "update_halo_kernel2_xvel_minus_2_left",
          "update_halo_kernel2_xvel_minus_4_right", "update_halo_kernel2_xvel_minus_2_right",
          "update_halo_kernel2_xvel_plus_4_back", "update_halo_kernel2_xvel_plus_2_back",
          "update_halo_kernel2_xvel_plus_4_front", "update_halo_kernel2_xvel_plus_2_front"}},
        {yvel0, FIELD_YVEL0, yvel1, FIELD_YVEL1,
         {"update_halo_kernel2_yvel_minus_4_bot", "update_halo_kernel2_yvel_minus_2_bot",
          "update_halo_kernel2_yvel_minus_4_top", "update_halo_kernel2_yvel_minus_2_top",
          "update_halo_kernel2_yvel_plus_4_left", "update_halo_kernel2_yvel_plus_2_left",
          "update_halo_kernel2_yvel_plus_4_right", "update_halo_kernel2_yvel_plus_2_right",
          "update_halo_kernel2_yvel_plus_4_back", "update_halo_kernel2_yvel_plus_2_back",
          "update_halo_kernel2_yvel_plus_4_front", "update_halo_kernel2_yvel_plus_2_front"}},
        {zvel0, FIELD_ZVEL0, zvel1, FIELD_ZVEL1,
         {"update_halo_kernel2_zvel_plus_4_bot", "update_halo_kernel2_zvel_plus_2_bot",
          "update_halo_kernel2_zvel_plus_4_top", "update_halo_kernel2_zvel_plus_2_top",
          "update_halo_kernel2_zvel_plus_4_left", "update_halo_kernel2_zvel_plus_2_left",
          "update_halo_kernel2_zvel_plus_4_right", "update_halo_kernel2_zvel_plus_2_right",
          "update_halo_kernel2_zvel_minus_4_back", "update_halo_kernel2_zvel_minus_2_back",
          "update_halo_kernel2_zvel_minus_4_front", "update_halo_kernel2_zvel_minus_2_front"}}};
    for (const Vel &v : vels) {
      auto K = [&](int i, std::vector<int> rng, int st) { k2(v.names[i], rng, v.a, v.fa, v.b, v.fb, st); };
      if (d == 2) K(0, R(x_min - d, x_max + 1 + d, y_min - 2, y_min - 1, z_min - d, z_max + 1 + d), S_0P40);
      K(1, R(x_min - d, x_max + 1 + d, y_min - 1, y_min, z_min - d, z_max + 1 + d), S_0P20);
      if (d == 2) K(2, R(x_min - d, x_max + 1 + d, y_max + 2, y_max + 3, z_min - d, z_max + 1 + d), S_0M40);
      K(3, R(x_min - d, x_max + 1 + d, y_max + 1, y_max + 2, z_min - d, z_max + 1 + d), S_0M20);
      if (d == 2) K(4, R(x_min - 2, x_min - 1, y_min - d, y_max + 1 + d, z_min - d, z_max + 1 + d), S_P400);
      K(5, R(x_min - 1, x_min, y_min - d, y_max + 1 + d, z_min - d, z_max + 1 + d), S_P200);
      if (d == 2) K(6, R(x_max + 2, x_max + 3, y_min - d, y_max + 1 + d, z_min - d, z_max + 1 + d), S_M400);
      K(7, R(x_max + 1, x_max + 2, y_min - d, y_max + 1 + d, z_min - d, z_max + 1 + d), S_M200);
      if (d == 2) K(8, R(x_min - d, x_max + 1 + d, y_min - d, y_max + 1 + d, z_min - 2, z_min - 1), S_00P4);
      K(9, R(x_min - d, x_max + 1 + d, y_min - d, y_max + 1 + d, z_min - 1, z_min), S_00P2);
      if (d == 2) K(10, R(x_min - d, x_max + 1 + d, y_min - d, y_max + 1 + d, z_max + 2, z_max + 3), S_00M4);
      K(11, R(x_min - d, x_max + 1 + d, y_min - d, y_max + 1 + d, z_max + 1, z_max + 2), S_00M2);
    }
    // x-face fluxes (kernel3)
    {
      auto K = [&](const char *k, std::vector<int> rng, int st) {
        k2(k, rng, vol_flux_x, FIELD_VOL_FLUX_X, mass_flux_x, FIELD_MASS_FLUX_X, st);
      };
      if (d == 2) K("update_halo_kernel3_plus_4_a", R(x_min - d, x_max + 1 + d, y_min - 2, y_min - 1, z_min - d, z_max + d), S_0P40);
      K("update_halo_kernel3_plus_2_a", R(x_min - d, x_max + 1 + d, y_min - 1, y_min, z_min - d, z_max + d), S_0P20);
      if (d == 2) K("update_halo_kernel3_plus_4_b", R(x_min - d, x_max + 1 + d, y_max + 1, y_max + 2, z_min - d, z_max + d), S_0M40);
      K("update_halo_kernel3_plus_2_b", R(x_min - d, x_max + 1 + d, y_max, y_max + 1, z_min - d, z_max + d), S_0M20);
      if (d == 2) K("update_halo_kernel3_minus_4_a", R(x_min - 2, x_min - 1, y_min - d, y_max + d, z_min - d, z_max + d), S_P400);
      K("update_halo_kernel3_minus_2_a", R(x_min - 1, x_min, y_min - d, y_max + d, z_min - d, z_max + d), S_P200);
      if (d == 2) K("update_halo_kernel3_minus_4_b", R(x_max + 2, x_max + 3, y_min - d, y_max + d, z_min - d, z_max + d), S_M400);
      K("update_halo_kernel3_minus_2_b", R(x_max + 1, x_max + 2, y_min - d, y_max + d, z_min - d, z_max + d), S_M200);
      if (d == 2) K("update_halo_kernel3_plus_4_back", R(x_min - d, x_max + d, y_min - d, y_max + d, z_min - 2, z_min - 1), S_00P4);
      K("update_halo_kernel3_plus_2_back", R(x_min - d, x_max + d, y_min - d, y_max + d, z_min - 1, z_min), S_00P2);
      if (d == 2) K("update_halo_kernel3_plus_4_front", R(x_min - d, x_max + d, y_min - d, y_max + d, z_max + 1, z_max + 2), S_00M4);
      K("update_halo_kernel3_plus_2_front", R(x_min - d, x_max + d, y_min - d, y_max + d, z_max, z_max + 1), S_00M2);
    }
    // y-face fluxes (kernel4)
    {
      auto K = [&](const char *k, std::vector<int> rng, int st) {
        k2(k, rng, vol_flux_y, FIELD_VOL_FLUX_Y, mass_flux_y, FIELD_MASS_FLUX_Y, st);
      };
      if (d == 2) K("update_halo_kernel4_minus_4_a", R(x_min - d, x_max + d, y_min - 2, y_min - 1, z_min - d, z_max + d), S_0P40);
      K("update_halo_kernel4_minus_2_a", R(x_min - d, x_max + d, y_min - 1, y_min, z_min - d, z_max + d), S_0P20);
      if (d == 2) K("update_halo_kernel4_minus_4_b", R(x_min - d, x_max + d, y_max + 2, y_max + 3, z_min - d, z_max + d), S_0M40);
      K("update_halo_kernel4_minus_2_b", R(x_min - d, x_max + d, y_max + 1, y_max + 2, z_min - d, z_max + d), S_0M20);
      if (d == 2) K("update_halo_kernel4_plus_4_a", R(x_min - 2, x_min - 1, y_min - d, y_max + 1 + d, z_min - d, z_max + d), S_P400);
      K("update_halo_kernel4_plus_2_a", R(x_min - 1, x_min, y_min - d, y_max + 1 + d, z_min - d, z_max + d), S_P200);
      if (d == 2) K("update_halo_kernel4_plus_4_b", R(x_max + 1, x_max + 2, y_min - d, y_max + 1 + d, z_min - d, z_max + d), S_M400);
      K("update_halo_kernel4_plus_2_b", R(x_max, x_max + 1, y_min - d, y_max + 1 + d, z_min - d, z_max + d), S_M200);
      if (d == 2) K("update_halo_kernel4_plus_4_back", R(x_min - d, x_max + d, y_min - d, y_max + d, z_min - 2, z_min - 1), S_00P4);
      K("update_halo_kernel4_plus_2_back", R(x_min - d, x_max + d, y_min - d, y_max + d, z_min - 1, z_min), S_00P2);
      if (d == 2) K("update_halo_kernel4_plus_4_front", R(x_min - d, x_max + d, y_min - d, y_max + d, z_max + 1, z_max + 2), S_00M4);
      K("update_halo_kernel4_plus_2_front", R(x_min - d, x_max + d, y_min - d, y_max + d, z_max, z_max + 1), S_00M2);
    }
    // z-face fluxes (kernel5)
    {
      auto K = [&](const char *k, std::vector<int> rng, int st) {
        k2(k, rng, vol_flux_z, FIELD_VOL_FLUX_Z, mass_flux_z, FIELD_MASS_FLUX_Z, st);
      };
      if (d == 2) K("update_halo_kernel5_plus_4_a", R(x_min - d, x_max + d, y_min - 2, y_min - 1, z_min - d, z_max + 1 + d), S_0P40);
      K("update_halo_kernel5_plus_2_a", R(x_min - d, x_max + d, y_min - 1, y_min, z_min - d, z_max + 1 + d), S_0P20);
      if (d == 2) K("update_halo_kernel5_plus_4_b", R(x_min - d, x_max + d, y_max + 1, y_max + 2, z_min - d, z_max + 1 + d), S_0M40);
      K("update_halo_kernel5_plus_2_b", R(x_min - d, x_max + d, y_max + 0, y_max + 1, z_min - d, z_max + 1 + d), S_0M20);
      if (d == 2) K("update_halo_kernel5_plus_4_left", R(x_min - 2, x_min - 1, y_min - d, y_max + d, z_min - d, z_max + 1 + d), S_P400);
      K("update_halo_kernel5_plus_2_left", R(x_min - 1, x_min, y_min - d, y_max + d, z_min - d, z_max + 1 + d), S_P200);
      if (d == 2) K("update_halo_kernel5_plus_4_right", R(x_max + 1, x_max + 2, y_min - d, y_max + d, z_min - d, z_max + 1 + d), S_M400);
      K("update_halo_kernel5_plus_2_right", R(x_max, x_max + 1, y_min - d, y_max + d, z_min - d, z_max + 1 + d), S_M200);
      if (d == 2) K("update_halo_kernel5_minus_4_back", R(x_min - d, x_max + d, y_min - d, y_max + d, z_min - 2, z_min - 1), S_00P4);
      K("update_halo_kernel5_minus_2_back", R(x_min - d, x_max + d, y_min - d, y_max + d, z_min - 1, z_min), S_00P2);
      if (d == 2) K("update_halo_kernel5_minus_4_front", R(x_min - d, x_max + d, y_min - d, y_max + d, z_max + 2, z_max + 3), S_00M4);
      K("update_halo_kernel5_minus_2_front", R(x_min - d, x_max + d, y_min - d, y_max + d, z_max + 1, z_max + 2), S_00M2);
    }
  }

  void field_summary() {  // field_summary.cpp:40-113
    int rng[6];
    ideal_gas(0);
    loop("field_summary_kernel", inner(rng),
         {dat(volume, S000, ACC_READ), dat(density0, S000, ACC_READ), dat(energy0, S000, ACC_READ),
          dat(pressure, S000, ACC_READ), dat(xvel0, S_fP1P1P1, ACC_READ), dat(yvel0, S_fP1P1P1, ACC_READ),
          dat(zvel0, S_fP1P1P1, ACC_READ), arg_reduce(red_vol, 1, ACC_INC), arg_reduce(red_mass, 1, ACC_INC),
          arg_reduce(red_ie, 1, ACC_INC), arg_reduce(red_ke, 1, ACC_INC), arg_reduce(red_press, 1, ACC_INC)});
    double vol = 0, mass = 0, ie = 0, ke = 0, press = 0;
    r.reduction_result(red_vol, &vol);
    r.reduction_result(red_mass, &mass);
    r.reduction_result(red_ie, &ie);
    r.reduction_result(red_ke, &ke);
    r.reduction_result(red_press, &press);
    double row[8] = {(double)step, clover_time, vol, mass, ie, ke, press, dt};
    summaries.insert(summaries.end(), row, row + 8);
  }

  void viscosity_func() {  // viscosity.cpp:38-62
    int rng[6];
    loop("viscosity_kernel", inner(rng),
         {dat(xvel0, S_fP1P1P1, ACC_READ), dat(yvel0, S_fP1P1P1, ACC_READ), dat(celldx, S_P100_STRID_X, ACC_READ),
          dat(celldy, S_0P10_STRID_Y, ACC_READ), dat(pressure, S_6PT, ACC_READ), dat(density0, S000, ACC_READ),
          dat(viscosity, S000, ACC_WRITE), dat(zvel0, S_fP1P1P1, ACC_READ), dat(celldz, S_00P1_STRID_Z, ACC_READ),
          dat(xarea, S000, ACC_READ), dat(yarea, S000, ACC_READ), dat(zarea, S000, ACC_READ)});
  }

  // calc_dt.cpp:39-145
  void calc_dt(double *local_dt, double *xl_pos, double *yl_pos, int *jldt, int *kldt) {
    int rng[6];
    double jk_control = 1.1;
    inner(rng);
    loop("calc_dt_kernel", rng,
         {dat(celldx, S_P100_STRID_X, ACC_READ), dat(celldy, S_0P10_STRID_Y, ACC_READ),
          dat(soundspeed, S000, ACC_READ), dat(viscosity, S000, ACC_READ), dat(density0, S000, ACC_READ),
          dat(xvel0, S_fP1P1P1, ACC_READ), dat(xarea, S000, ACC_READ), dat(volume, S000, ACC_READ),
          dat(yvel0, S_fP1P1P1, ACC_READ), dat(yarea, S000, ACC_READ), dat(work_array1, S000, ACC_WRITE),
          dat(celldz, S_00P1_STRID_Z, ACC_READ), dat(zvel0, S_fP1P1P1, ACC_READ), dat(zarea, S000, ACC_READ)});
    loop("calc_dt_kernel_min", rng, {dat(work_array1, S000, ACC_READ), arg_reduce(red_local_dt, 1, ACC_MIN)});
    jk_control = jk_control - (jk_control - (int)(jk_control));
    *jldt = ((int)jk_control) % (field.x_max - 2);
    *kldt = 1 + (jk_control / (field.x_max - 2));
    int lldt = 1 + (jk_control / (field.x_max - 2));
    int getpoint[] = {*jldt - 1 + 2, *jldt + 2, *kldt - 1 + 2, *kldt + 2, lldt - 1 + 2, lldt + 2};
    loop("calc_dt_kernel_get", "calc_dt_kernel_getx", getpoint,
         {dat(cellx, S_STRID_X, ACC_READ), dat(celly, S_STRID_Y, ACC_READ), arg_reduce(red_xl_pos, 1, ACC_INC),
          arg_reduce(red_yl_pos, 1, ACC_INC), dat(cellz, S_STRID_Z, ACC_READ), arg_reduce(red_zl_pos, 1, ACC_INC)});
    r.reduction_result(red_local_dt, local_dt);
    r.reduction_result(red_xl_pos, xl_pos);
    r.reduction_result(red_yl_pos, yl_pos);
    *local_dt = op_min(*local_dt, g_big);
    if (*local_dt < dtmin) throw Error(E_STATE, "cloverleaf3d: timestep below dtmin (calc_dt.cpp:104-140)");
  }

  // time_step.cpp:37-151
  void timestep() {
    double dtlp, xl_pos = 0.0, yl_pos = 0.0;
    int jldt, kldt;
    ideal_gas(0);
    set_fields({FIELD_DENSITY0, FIELD_ENERGY0, FIELD_PRESSURE, FIELD_XVEL0, FIELD_YVEL0});
    update_halo(fields, 1);
    viscosity_func();
    set_fields({FIELD_VISCOSITY});
    update_halo(fields, 1);
    calc_dt(&dtlp, &xl_pos, &yl_pos, &jldt, &kldt);
    double dt_temp = g_big;
    if (dtlp <= dt_temp) {
      dt_temp = dtlp;
      jdt = jldt;
      kdt = kldt;
    }
    dt_temp = op_min(op_min(dt_temp, (dtold * dtrise)), dtmax);
    r.decl_const("cloverleaf3d/dt", 1, "double", &dt_temp);
    dt = dt_temp;
    if (dt < dtmin) throw Error(E_STATE, "cloverleaf3d: small timestep (time_step.cpp:142-145)");
    dtold = dt;
  }

  void revert() {  // revert.cpp:39-63
    int rng[6];
    loop("revert_kernel", inner(rng),
         {dat(density0, S000, ACC_READ), dat(density1, S000, ACC_WRITE), dat(energy0, S000, ACC_READ),
          dat(energy1, S000, ACC_WRITE)});
  }

  // PdV.cpp:40-134. The predictor's halo update sets only the flags the
  // reference assigns there; the z velocity, z flux and sound speed flags
  // keep their previous values.
  void PdV(int predict) {
    int rng[6];
    inner(rng);
    if (predict) {
      loop("PdV_kernel_predict", rng,
           {dat(xarea, S_P100, ACC_READ), dat(xvel0, S_fP1P1P1, ACC_READ), dat(yarea, S_0P10, ACC_READ),
            dat(yvel0, S_fP1P1P1, ACC_READ), dat(work_array1, S000, ACC_WRITE), dat(volume, S000, ACC_READ),
            dat(pressure, S000, ACC_READ), dat(density0, S000, ACC_READ), dat(density1, S000, ACC_WRITE),
            dat(viscosity, S000, ACC_READ), dat(energy0, S000, ACC_READ), dat(energy1, S000, ACC_WRITE),
            dat(zarea, S_00P1, ACC_READ), dat(zvel0, S_fP1P1P1, ACC_READ)});
    } else {
      loop("PdV_kernel_nopredict", rng,
           {dat(xarea, S_P100, ACC_READ), dat(xvel0, S_fP1P1P1, ACC_READ), dat(xvel1, S_fP1P1P1, ACC_READ),
            dat(yarea, S_0P10, ACC_READ), dat(yvel0, S_fP1P1P1, ACC_READ), dat(yvel1, S_fP1P1P1, ACC_READ),
            dat(work_array1, S000, ACC_WRITE), dat(volume, S000, ACC_READ), dat(pressure, S000, ACC_READ),
            dat(density0, S000, ACC_READ), dat(density1, S000, ACC_WRITE), dat(viscosity, S000, ACC_READ),
            dat(energy0, S000, ACC_READ), dat(energy1, S000, ACC_WRITE), dat(zarea, S_00P1, ACC_READ),
            dat(zvel0, S_fP1P1P1, ACC_READ), dat(zvel1, S_fP1P1P1, ACC_READ)});
    }
    if (predict) {
      ideal_gas(1);
      for (int fld : {FIELD_DENSITY0, FIELD_ENERGY0, FIELD_VISCOSITY, FIELD_DENSITY1, FIELD_ENERGY1, FIELD_XVEL0,
                      FIELD_YVEL0, FIELD_XVEL1, FIELD_YVEL1, FIELD_VOL_FLUX_X, FIELD_VOL_FLUX_Y, FIELD_MASS_FLUX_X,
                      FIELD_MASS_FLUX_Y})
        fields[fld] = 0;
      fields[FIELD_PRESSURE] = 1;
      update_halo(fields, 1);
      revert();
    }
  }

  void accelerate() {  // accelerate.cpp:38-68
    int rng[6];
    loop("accelerate_kernel", inner(rng, 1, 1, 1),
         {dat(density0, S_fM1M1M1, ACC_READ), dat(volume, S_fM1M1M1, ACC_READ), dat(work_array1, S000, ACC_WRITE),
          dat(xvel0, S000, ACC_READ), dat(xvel1, S000, ACC_WRITE), dat(xarea, S_f0M1M1, ACC_READ),
          dat(pressure, S_fM1M1M1, ACC_READ), dat(yvel0, S000, ACC_READ), dat(yvel1, S000, ACC_WRITE),
          dat(yarea, S_fM10M1, ACC_READ), dat(viscosity, S_fM1M1M1, ACC_READ), dat(zvel0, S000, ACC_READ),
          dat(zvel1, S000, ACC_WRITE), dat(zarea, S_fM1M10, ACC_READ)});
  }

  void flux_calc() {  // flux_calc.cpp:38-77
    int rng[6];
    loop("flux_calc_kernelx", inner(rng, 1, 0, 0),
         {dat(vol_flux_x, S000, ACC_WRITE), dat(xarea, S000, ACC_READ), dat(xvel0, S_f0P1P1, ACC_READ),
          dat(xvel1, S_f0P1P1, ACC_READ)});
    loop("flux_calc_kernely", inner(rng, 0, 1, 0),
         {dat(vol_flux_y, S000, ACC_WRITE), dat(yarea, S000, ACC_READ), dat(yvel0, S_fP10P1, ACC_READ),
          dat(yvel1, S_fP10P1, ACC_READ)});
    loop("flux_calc_kernelz", inner(rng, 0, 0, 1),
         {dat(vol_flux_z, S000, ACC_WRITE), dat(zarea, S000, ACC_READ), dat(zvel0, S_fP1P10, ACC_READ),
          dat(zvel1, S_fP1P10, ACC_READ)});
  }

  // advec_cell.cpp:40-252
  void advec_cell(int sweep_number, int dir) {
    const int x_min = field.x_min, x_max = field.x_max, y_min = field.y_min, y_max = field.y_max;
    const int z_min = field.z_min, z_max = field.z_max;
    int rangexyz[] = {x_min - 2, x_max + 2, y_min - 2, y_max + 2, z_min - 2, z_max + 2};
    int inner_r[] = {x_min, x_max, y_min, y_max, z_min, z_max};
    int plus2x[] = {x_min, x_max + 2, y_min, y_max, z_min, z_max};
    int plus2yz[] = {x_min, x_max, y_min, y_max + 2, z_min, z_max + 2};
    int plus2z[] = {x_min, x_max, y_min, y_max, z_min, z_max + 2};
    auto kernel4 = [&](const char *k, int mass_flux, int vol_flux, int st) {
      loop(k, inner_r,
           {dat(density1, S000, ACC_RW), dat(energy1, S000, ACC_RW), dat(mass_flux, st, ACC_READ),
            dat(vol_flux, st, ACC_READ), dat(work_array1, S000, ACC_READ), dat(work_array2, S000, ACC_READ),
            dat(work_array3, S000, ACC_WRITE), dat(work_array4, S000, ACC_WRITE), dat(work_array5, S000, ACC_WRITE),
            dat(work_array6, S000, ACC_WRITE), dat(work_array7, st, ACC_READ)});
    };
    if (dir == G_XDIR) {
      if (sweep_number == 1)
        loop("advec_cell_kernel1_xdir", rangexyz,
             {dat(work_array1, S000, ACC_WRITE), dat(work_array2, S000, ACC_WRITE), dat(volume, S000, ACC_READ),
              dat(vol_flux_x, S_P100, ACC_READ), dat(vol_flux_y, S_0P10, ACC_READ), dat(vol_flux_z, S_00P1, ACC_READ)});
      else if (sweep_number == 3)
        loop("advec_cell_kernel2_xdir", rangexyz,
             {dat(work_array1, S000, ACC_WRITE), dat(work_array2, S000, ACC_WRITE), dat(volume, S000, ACC_READ),
              dat(vol_flux_x, S_P100, ACC_READ)});
      loop("advec_cell_kernel3_xdir", plus2x,
           {dat(vol_flux_x, S000, ACC_READ), dat(work_array1, S_M100, ACC_READ), dat(xx, S_P100_STRID_X, ACC_READ),
            dat(vertexdx, S_P100_M100_STRID_X, ACC_READ), dat(density1, S_P100_M100_M200, ACC_READ),
            dat(energy1, S_P100_M100_M200, ACC_READ), dat(mass_flux_x, S000, ACC_WRITE),
            dat(work_array7, S000, ACC_WRITE)});
      kernel4("advec_cell_kernel4_xdir", mass_flux_x, vol_flux_x, S_P100);
    } else if (dir == G_YDIR) {
      if (sweep_number == 2) {
        if (advect_x)
          loop("advec_cell_kernel1_ydir", rangexyz,
               {dat(work_array1, S000, ACC_WRITE), dat(work_array2, S000, ACC_WRITE), dat(volume, S000, ACC_READ),
                dat(vol_flux_z, S_00P1, ACC_READ), dat(vol_flux_y, S_0P10, ACC_READ)});
        else
          loop("advec_cell_kernel2_ydir", rangexyz,
               {dat(work_array1, S000, ACC_WRITE), dat(work_array2, S000, ACC_WRITE), dat(volume, S000, ACC_READ),
                dat(vol_flux_y, S_0P10, ACC_READ), dat(vol_flux_x, S_P100, ACC_READ)});
      }
      loop("advec_cell_kernel3_ydir", plus2yz,
           {dat(vol_flux_y, S000, ACC_READ), dat(work_array1, S_0M10, ACC_READ), dat(yy, S_0P10_STRID_Y, ACC_READ),
            dat(vertexdy, S_0P10_0M10_STRID_Y, ACC_READ), dat(density1, S_0P10_0M10_0M20, ACC_READ),
            dat(energy1, S_0P10_0M10_0M20, ACC_READ), dat(mass_flux_y, S000, ACC_WRITE),
            dat(work_array7, S000, ACC_WRITE)});
      kernel4("advec_cell_kernel4_ydir", mass_flux_y, vol_flux_y, S_0P10);
    } else if (dir == G_ZDIR) {
      if (sweep_number == 1)
        loop("advec_cell_kernel1_zdir", rangexyz,
             {dat(work_array1, S000, ACC_WRITE), dat(work_array2, S000, ACC_WRITE), dat(volume, S000, ACC_READ),
              dat(vol_flux_x, S_P100, ACC_READ), dat(vol_flux_y, S_0P10, ACC_READ), dat(vol_flux_z, S_00P1, ACC_READ)});
      else if (sweep_number == 3)
        loop("advec_cell_kernel2_zdir", rangexyz,
             {dat(work_array1, S000, ACC_WRITE), dat(work_array2, S000, ACC_WRITE), dat(volume, S000, ACC_READ),
              dat(vol_flux_z, S_00P1, ACC_READ)});
      loop("advec_cell_kernel3_zdir", plus2z,
           {dat(vol_flux_z, S000, ACC_READ), dat(work_array1, S_00M1, ACC_READ), dat(zz, S_00P1_STRID_Z, ACC_READ),
            dat(vertexdz, S_00P1_00M1_STRID_Z, ACC_READ), dat(density1, S_00P1_00M1_00M2, ACC_READ),
            dat(energy1, S_00P1_00M1_00M2, ACC_READ), dat(mass_flux_z, S000, ACC_WRITE),
            dat(work_array7, S000, ACC_WRITE)});
      kernel4("advec_cell_kernel4_zdir", mass_flux_z, vol_flux_z, S_00P1);
    }
  }

  // advec_mom.cpp:40-290
  void advec_mom(int which_vel, int sweep_number, int dir) {
    const int x_min = field.x_min, x_max = field.x_max, y_min = field.y_min, y_max = field.y_max;
    const int z_min = field.z_min, z_max = field.z_max;
    int rangexyz[] = {x_min - 2, x_max + 2, y_min - 2, y_max + 2, z_min - 2, z_max + 2};
    int vel1 = which_vel == 1 ? xvel1 : which_vel == 2 ? yvel1 : zvel1;
    auto pre = [&](const char *k, std::initializer_list<Arg> fluxes) {
      std::vector<Arg> a = {dat(work_array6, S000, ACC_WRITE), dat(work_array7, S000, ACC_WRITE),
                            dat(volume, S000, ACC_READ)};
      a.insert(a.end(), fluxes.begin(), fluxes.end());
      r.par_loop(loops.get(k), k, clover_grid, 3, rangexyz, a.data(), (int)a.size());
    };
    if (sweep_number == 1 && dir == 1)
      pre("advec_mom_kernel_x1", {dat(vol_flux_x, S_P100, ACC_READ), dat(vol_flux_y, S_0P10, ACC_READ),
                                  dat(vol_flux_z, S_00P1, ACC_READ)});
    else if (sweep_number == 1 && dir == 3)
      pre("advec_mom_kernel_z1", {dat(vol_flux_x, S_P100, ACC_READ), dat(vol_flux_y, S_0P10, ACC_READ),
                                  dat(vol_flux_z, S_00P1, ACC_READ)});
    else if (sweep_number == 2 && advect_x)
      pre("advec_mom_kernel_x2", {dat(vol_flux_y, S_0P10, ACC_READ), dat(vol_flux_z, S_00P1, ACC_READ)});
    else if (sweep_number == 2 && !advect_x)
      pre("advec_mom_kernel_y2", {dat(vol_flux_x, S_P100, ACC_READ), dat(vol_flux_y, S_0P10, ACC_READ)});
    else if (sweep_number == 3 && dir == 1)
      pre("advec_mom_kernel_x3", {dat(vol_flux_x, S_P100, ACC_READ)});
    else if (sweep_number == 3 && dir == 3)
      pre("advec_mom_kernel_z3", {dat(vol_flux_z, S_00P1, ACC_READ)});
    int part2[] = {x_min, x_max + 1, y_min, y_max + 1, z_min, z_max + 1};
    if (dir == 1) {
      if (which_vel == 1) {
        int r1[] = {x_min - 2, x_max + 2, y_min, y_max + 1, z_min, z_max + 1};
        loop("advec_mom_kernel_mass_flux_x", r1,
             {dat(work_array1, S000, ACC_WRITE), dat(mass_flux_x, S_fP1M1M1, ACC_READ)});
        int r2[] = {x_min - 1, x_max + 2, y_min, y_max + 1, z_min, z_max + 1};
        loop("advec_mom_kernel_post_pre_advec_x", r2,
             {dat(work_array2, S000, ACC_WRITE), dat(work_array7, S_fM1M1M1, ACC_READ),
              dat(density1, S_fM1M1M1, ACC_READ), dat(work_array3, S000, ACC_WRITE),
              dat(work_array1, S_M100, ACC_READ)});
      }
      int r3[] = {x_min - 1, x_max + 1, y_min, y_max + 1, z_min, z_max + 1};
      loop("advec_mom_kernel1_x_nonvector", "advec_mom_kernel1_x", r3,
           {dat(work_array1, S000, ACC_READ), dat(work_array3, S_P100, ACC_READ), dat(work_array5, S000, ACC_WRITE),
            dat(celldx, S_P100_M100_STRID_X, ACC_READ), dat(vel1, S_P100_P200_M100, ACC_READ)});
      loop("advec_mom_kernel2_x", part2,
           {dat(vel1, S000, ACC_RW), dat(work_array2, S000, ACC_READ), dat(work_array3, S000, ACC_READ),
            dat(work_array5, S_M100, ACC_READ)});
    } else if (dir == 2) {
      if (which_vel == 1) {
        int r1[] = {x_min, x_max + 1, y_min - 2, y_max + 2, z_min, z_max + 1};
        loop("advec_mom_kernel_mass_flux_y", r1,
             {dat(work_array1, S000, ACC_WRITE), dat(mass_flux_y, S_fM1P1M1, ACC_READ)});
        int r2[] = {x_min, x_max + 1, y_min - 1, y_max + 2, z_min, z_max + 1};
        loop("advec_mom_kernel_post_pre_advec_y", r2,
             {dat(work_array2, S000, ACC_WRITE), dat(work_array7, S_fM1M1M1, ACC_READ),
              dat(density1, S_fM1M1M1, ACC_READ), dat(work_array3, S000, ACC_WRITE),
              dat(work_array1, S_0M10, ACC_READ)});
      }
      int r3[] = {x_min, x_max + 1, y_min - 1, y_max + 1, z_min, z_max + 1};
      loop("advec_mom_kernel1_y_nonvector", "advec_mom_kernel1_y", r3,
           {dat(work_array1, S000, ACC_READ), dat(work_array3, S_0P10, ACC_READ), dat(work_array5, S000, ACC_WRITE),
            dat(celldy, S_0P10_0M10_STRID_Y, ACC_READ), dat(vel1, S_0P10_0P20_0M10, ACC_READ)});
      loop("advec_mom_kernel2_y", part2,
           {dat(vel1, S000, ACC_RW), dat(work_array2, S000, ACC_READ), dat(work_array3, S000, ACC_READ),
            dat(work_array5, S_0M10, ACC_READ)});
    } else if (dir == 3) {
      if (which_vel == 1) {
        int r1[] = {x_min, x_max + 1, y_min, y_max + 1, z_min - 2, z_max + 2};
        loop("advec_mom_kernel_mass_flux_z", r1,
             {dat(work_array1, S000, ACC_WRITE), dat(mass_flux_z, S_fM1M1P1, ACC_READ)});
        int r2[] = {x_min, x_max + 1, y_min, y_max + 1, z_min - 1, z_max + 2};
        loop("advec_mom_kernel_post_pre_advec_z", r2,
             {dat(work_array2, S000, ACC_WRITE), dat(work_array7, S_fM1M1M1, ACC_READ),
              dat(density1, S_fM1M1M1, ACC_READ), dat(work_array3, S000, ACC_WRITE),
              dat(work_array1, S_00M1, ACC_READ)});
      }
      int r3[] = {x_min, x_max + 1, y_min, y_max + 1, z_min - 1, z_max + 1};
      loop("advec_mom_kernel1_z_nonvector", "advec_mom_kernel1_z", r3,
           {dat(work_array1, S000, ACC_READ), dat(work_array3, S_00P1, ACC_READ), dat(work_array5, S000, ACC_WRITE),
            dat(celldz, S_00P1_00M1_STRID_Z, ACC_READ), dat(vel1, S_00P1_00P2_00M1, ACC_READ)});
      loop("advec_mom_kernel2_z", part2,
           {dat(vel1, S000, ACC_RW), dat(work_array2, S000, ACC_READ), dat(work_array3, S000, ACC_READ),
            dat(work_array5, S_00M1, ACC_READ)});
    }
  }

  // advection.cpp:37-203
  void advection() {
    int sweep_number = 1;
    int direction = advect_x ? G_XDIR : G_ZDIR;
    auto mom_fields = [&](int dir) {
      set_fields({FIELD_DENSITY1, FIELD_ENERGY1, FIELD_XVEL1, FIELD_YVEL1, FIELD_ZVEL1});
      fields[FIELD_MASS_FLUX_X] = (dir == G_XDIR);
      fields[FIELD_MASS_FLUX_Y] = (dir == G_YDIR);
      fields[FIELD_MASS_FLUX_Z] = (dir == G_ZDIR);
      update_halo(fields, 2);
      advec_mom(G_XDIR, sweep_number, dir);
      advec_mom(G_YDIR, sweep_number, dir);
      advec_mom(G_ZDIR, sweep_number, dir);
    };
    set_fields({FIELD_DENSITY1, FIELD_ENERGY1, FIELD_VOL_FLUX_X, FIELD_VOL_FLUX_Y, FIELD_VOL_FLUX_Z});
    update_halo(fields, 2);
    advec_cell(sweep_number, direction);
    mom_fields(direction);
    sweep_number = 2;
    direction = G_YDIR;
    set_fields({FIELD_DENSITY1, FIELD_ENERGY1, FIELD_VOL_FLUX_X, FIELD_VOL_FLUX_Y, FIELD_VOL_FLUX_Z});
    update_halo(fields, 2);
    advec_cell(sweep_number, direction);
    mom_fields(direction);
    sweep_number = 3;
    direction = advect_x ? G_ZDIR : G_XDIR;
    advec_cell(sweep_number, direction);
    mom_fields(direction);
  }

  void reset_field() {  // reset_field.cpp:38-70
    int rng[6];
    loop("reset_field_kernel1", inner(rng),
         {dat(density0, S000, ACC_WRITE), dat(density1, S000, ACC_READ), dat(energy0, S000, ACC_WRITE),
          dat(energy1, S000, ACC_READ)});
    loop("reset_field_kernel2", inner(rng, 1, 1, 1),
         {dat(xvel0, S000, ACC_WRITE), dat(xvel1, S000, ACC_READ), dat(yvel0, S000, ACC_WRITE),
          dat(yvel1, S000, ACC_READ), dat(zvel0, S000, ACC_WRITE), dat(zvel1, S000, ACC_READ)});
  }

  // clover_leaf.cpp:133-169 + start.cpp:37-100
  void setup(const ops_b200_clover3d_deck &deck) {
    read_input(deck);
    const char *P = "cloverleaf3d/";
    auto C = [&](const char *n, int dim, const char *type, const void *p) {
      r.decl_const((std::string(P) + n).c_str(), dim, type, p);
    };
    C("g_small", 1, "double", &g_small);
    C("g_big", 1, "double", &g_big);
    C("dtc_safe", 1, "double", &dtc_safe);
    C("dtu_safe", 1, "double", &dtu_safe);
    C("dtv_safe", 1, "double", &dtv_safe);
    C("dtw_safe", 1, "double", &dtw_safe);
    C("dtdiv_safe", 1, "double", &dtdiv_safe);
    C("field", 1, "field_type", &field);
    C("grid", 1, "grid_type", &grid);
    C("states", number_of_states, "state_type", states);
    C("number_of_states", 1, "int", &number_of_states);
    C("g_sphe", 1, "int", &g_sphe);
    C("g_point", 1, "int", &g_point);
    C("g_cube", 1, "int", &g_cube);
    C("dt", 1, "double", &dt);
    clover_time = 0.0;
    step = 0;
    dtold = dtinit;
    dt = dtinit;
    build_field();
    r.partition("3D_BLOCK_DECOMPOSE");  // build_field.cpp:318
    initialise_chunk();
    generate();
    advect_x = 1;
    ideal_gas(0);
    set_fields({FIELD_DENSITY0, FIELD_ENERGY0, FIELD_PRESSURE, FIELD_VISCOSITY, FIELD_DENSITY1, FIELD_ENERGY1,
                FIELD_XVEL0, FIELD_YVEL0, FIELD_ZVEL0, FIELD_XVEL1, FIELD_YVEL1, FIELD_ZVEL1});
    update_halo(fields, 2);
    field_summary();
  }

  // One hydro cycle (clover_leaf.cpp:176-210). Returns true when complete.
  bool cycle() {
    step = step + 1;
    timestep();
    PdV(1);
    accelerate();
    PdV(0);
    flux_calc();
    advection();
    reset_field();
    advect_x = advect_x ? 0 : 1;
    clover_time = clover_time + dt;
    if (summary_frequency != 0)
      if ((step % summary_frequency) == 0) field_summary();
    if ((clover_time + g_small) > end_time || (step >= end_step)) {
      complete = 1;
      field_summary();
      return true;
    }
    return false;
  }
};

}  // namespace clover3d
}  // namespace opsb

extern "C" int ops_b200_app_cloverleaf3d(const ops_b200_clover3d_deck *deck, int warmup_steps, double *summaries,
                                         int max_summaries, int *n_summaries, double *device_seconds,
                                         const char *dump_dir) {
  using namespace opsb;
  return capi_guard([&] {
    if (!deck || warmup_steps < 0) throw Error(E_ARG, "bad CloverLeaf 3D arguments");
    if (deck->x_cells < 2 || deck->y_cells < 2 || deck->z_cells < 2)
      throw Error(E_ARG, "x_cells, y_cells and z_cells must be >= 2");
    Runtime &r = Runtime::get();
    if (!r.initialized()) r.init(0, 0);
    ReleaseScope scope(r);
    const Runtime::Mark &mk = scope.mark();
    clover3d::Clover3D c(r);
    c.setup(*deck);
    EventPair ev;
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    bool started = false;
    if (warmup_steps == 0) {
      r.execute();
      OPSB_CUDA(cudaEventRecord(e0, r.stream()));
      started = true;
    }
    while (true) {
      bool done = c.cycle();
      if (!started && c.step == warmup_steps) {
        r.execute();
        OPSB_CUDA(cudaEventRecord(e0, r.stream()));
        started = true;
      }
      if (done) break;
    }
    r.execute();
    OPSB_CUDA(cudaEventRecord(e1, r.stream()));
    if (!started) OPSB_CUDA(cudaEventRecord(e0, r.stream()));
    OPSB_CUDA(cudaEventSynchronize(e1));
    if (device_seconds) *device_seconds = ev.ms() * 1e-3;
    int n = (int)(c.summaries.size() / 8);
    if (n_summaries) *n_summaries = n;
    if (summaries) memcpy(summaries, c.summaries.data(), sizeof(double) * 8 * std::min(n, max_summaries));
    if (dump_dir) {
      for (int i = mk.dats; i < r.ndats(); i++) {
        Dat &d = r.dat(i);
        std::vector<char> buf(r.dat_data_bytes(i));  // the rank's owned part when partitioned
        r.dat_fetch_data(i, buf.data(), buf.size());
        std::string path = std::string(dump_dir) + "/" + d.name + ".bin";
        FILE *f = fopen(path.c_str(), "wb");
        if (!f) throw Error(E_ARG, "cannot write " + path);
        fwrite(buf.data(), 1, buf.size(), f);
        fclose(f);
      }
    }
    scope.release();
    return 0;
  });
}
