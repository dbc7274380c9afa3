// CloverLeaf 2D driver on the OPS-B200 runtime: the loop sequence of the
// reference app (apps/c/CloverLeaf/clover_leaf.cpp:161-214 and the files it
// calls, cited per function), with the input deck passed as a struct
// instead of clover.in. Every ops_par_loop keeps the reference's kernel,
// range, stencils and access modes.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/ops_b200.h"
#include "clover_common.h"
#include "runtime.h"

namespace opsb {
int capi_guard(const std::function<int()> &f);

namespace clover {

struct Clover {
  Runtime &r;
  // run-time constants and state (clover_leaf.cpp:73-131)
  double g_small = 1.0e-16, g_big = 1.0e+21;
  double dtold = 0, dt = 0, clover_time = 0, dtinit = 0.1, dtmin = 0.0000001, dtmax = 1.0, dtrise = 1.5;
  double dtu_safe = 0.5, dtv_safe = 0.5, dtc_safe = 0.7, dtdiv_safe = 0.7;
  double end_time = 10.0;
  int end_step = 640000, summary_frequency = 10;
  int step = 0, advect_x = 1, complete = 0;
  int g_rect = G_RECT, g_circ = G_CIRC, g_point = G_POINT;
  int number_of_states = 0;
  state_type states[kMaxStates];
  grid_type grid;
  field_type field;
  int fields[NUM_FIELDS] = {0};
  int jdt = 0, kdt = 0;

  int clover_grid = -1;
  int density0, density1, energy0, energy1, pressure, viscosity, soundspeed, volume;
  int xvel0, xvel1, yvel0, yvel1, vol_flux_x, vol_flux_y, mass_flux_x, mass_flux_y, xarea, yarea;
  int work_array1, work_array2, work_array3, work_array4, work_array5, work_array6, work_array7;
  int cellx, celly, vertexx, vertexy, celldx, celldy, vertexdx, vertexdy, xx, yy;

  int S2D_00, S2D_00_P10, S2D_00_0P1, S2D_00_M10, S2D_00_0M1, S2D_00_P10_M10, S2D_00_0P1_0M1;
  int S2D_00_M10_M20, S2D_00_0M1_0M2, S2D_00_P20, S2D_00_0P2, S2D_00_M20, S2D_00_0M2;
  int S2D_00_P30, S2D_00_0P3, S2D_00_M30, S2D_00_0M3, S2D_00_P40, S2D_00_0P4, S2D_00_M40, S2D_00_0M4;
  int S2D_00_P10_0P1_P1P1, S2D_00_M10_0M1_M1M1, S2D_00_P10_0M1_P1M1, S2D_00_0P1_M10_M1P1, S2D_10_M10_01_0M1;
  int S2D_00_P10_M10_M20, S2D_00_P10_M10_STRID2D_X, S2D_00_0P1_0M1_0M2, S2D_00_0P1_0M1_STRID2D_Y;
  int S2D_00_P10_P20_M10, S2D_00_0P1_0P2_0M1, S2D_00_STRID2D_X, S2D_00_STRID2D_Y;
  int S2D_00_P10_STRID2D_X, S2D_00_0P1_STRID2D_Y, S2D_00_M10_STRID2D_X, S2D_00_0M1_STRID2D_Y;
  int red_local_dt, red_xl_pos, red_yl_pos, red_vol, red_mass, red_ie, red_ke, red_press, red_output;

  std::vector<double> summaries;  // per field_summary: step, time, vol, mass, ie, ke, press, dt

  explicit Clover(Runtime &rt) : r(rt) {
    memset(states, 0, sizeof(states));
    memset(&grid, 0, sizeof(grid));
    memset(&field, 0, sizeof(field));
  }

  PrefixedLoops loops{"cloverleaf/"};
  void loop(const char *k, const char *name, const int *range, std::initializer_list<Arg> a) {
    r.par_loop(loops.get(k), name, clover_grid, 2, range, a.begin(), (int)a.size());
  }
  Arg dat(int d, int s, int acc) { return arg_dat(d, 1, s, acc); }
  Arg dat_opt(int d, int s, int acc, int flag) { return arg_dat_opt(d, 1, s, acc, flag); }

  // read_input.cpp:36-276 (deck values already parsed by the caller).
  void read_input(const ops_b200_clover_deck &d) {
    grid.xmin = d.xmin; grid.ymin = d.ymin; grid.xmax = d.xmax; grid.ymax = d.ymax;
    grid.x_cells = d.x_cells; grid.y_cells = d.y_cells;
    dtinit = d.initial_timestep; dtmax = d.max_timestep; dtrise = d.timestep_rise;
    end_time = d.end_time; end_step = d.end_step; summary_frequency = d.summary_frequency;
    number_of_states = d.number_of_states;
    if (number_of_states < 1 || number_of_states > 16) throw Error(E_ARG, "1..16 states are supported");
    for (int i = 0; i < number_of_states; i++) {
      const ops_b200_clover_state &s = d.states[i];
      states[i].defined = 1;
      states[i].density = s.density; states[i].energy = s.energy;
      states[i].xvel = s.xvel; states[i].yvel = s.yvel;
      states[i].geometry = s.geometry;
      states[i].xmin = s.xmin; states[i].xmax = s.xmax; states[i].ymin = s.ymin; states[i].ymax = s.ymax;
      states[i].radius = s.radius;
    }
    field.x_min = 0 + 2; field.y_min = 0 + 2;
    field.x_max = grid.x_cells + 2; field.y_max = grid.y_cells + 2;
    field.left = 0; field.bottom = 0;
    // read_input.cpp:265-275: the state boxes shrink by 1 % of a cell, with
    // the cell width rounded to single precision as the reference does.
    float dx = (grid.xmax - grid.xmin) / (float)(grid.x_cells);
    float dy = (grid.ymax - grid.ymin) / (float)(grid.y_cells);
    for (int i = 0; i < number_of_states; i++) {
      states[i].xmin = states[i].xmin + (dx / 100.00);
      states[i].ymin = states[i].ymin + (dy / 100.00);
      states[i].xmax = states[i].xmax - (dx / 100.00);
      states[i].ymax = states[i].ymax - (dy / 100.00);
    }
  }

  int stencil(int points, std::initializer_list<int> offs, const char *name) {
    std::vector<int> o(offs);
    return r.decl_stencil(2, points, o.data(), nullptr, name);
  }
  int strided(int points, std::initializer_list<int> offs, std::initializer_list<int> stride, const char *name) {
    std::vector<int> o(offs), s(stride);
    return r.decl_stencil(2, points, o.data(), s.data(), name);
  }

  // build_field.cpp:35-239
  void build_field() {
    const int x_cells = grid.x_cells, y_cells = grid.y_cells;
    clover_grid = r.decl_block(2, "clover grid");
    int d_p[2] = {2, 2}, d_m[2] = {-2, -2}, base[2] = {0, 0};
    int size[2] = {x_cells + 5, y_cells + 5};
    auto D = [&](const char *n) { return r.decl_dat(clover_grid, 1, size, base, d_m, d_p, nullptr, 8, "double", n); };
    density0 = D("density0"); density1 = D("density1"); energy0 = D("energy0"); energy1 = D("energy1");
    pressure = D("pressure"); viscosity = D("viscosity"); soundspeed = D("soundspeed"); volume = D("volume");
    size[0]++; size[1]++;
    xvel0 = D("xvel0"); xvel1 = D("xvel1"); yvel0 = D("yvel0"); yvel1 = D("yvel1");
    work_array1 = D("work_array1"); work_array2 = D("work_array2"); work_array3 = D("work_array3");
    work_array4 = D("work_array4"); work_array5 = D("work_array5"); work_array6 = D("work_array6");
    work_array7 = D("work_array7");
    size[0] = x_cells + 6; size[1] = y_cells + 5;
    vol_flux_x = D("vol_flux_x"); mass_flux_x = D("mass_flux_x"); xarea = D("xarea");
    size[0] = x_cells + 5; size[1] = y_cells + 6;
    vol_flux_y = D("vol_flux_y"); mass_flux_y = D("mass_flux_y"); yarea = D("yarea");
    auto D1 = [&](int sx, int sy, int mx, int my, int px, int py, const char *type, const char *n) {
      int sz[2] = {sx, sy}, dm[2] = {mx, my}, dp[2] = {px, py};
      return r.decl_dat(clover_grid, 1, sz, base, dm, dp, nullptr, 0, type, n);
    };
    cellx = D1(x_cells + 5, 1, -2, 0, 2, 0, "double", "cellx");
    celldx = D1(x_cells + 5, 1, -2, 0, 2, 0, "double", "celldx");
    celly = D1(1, y_cells + 5, 0, -2, 0, 2, "double", "celly");
    celldy = D1(1, y_cells + 5, 0, -2, 0, 2, "double", "celldy");
    vertexx = D1(x_cells + 6, 1, -2, 0, 2, 0, "double", "vertexx");
    vertexdx = D1(x_cells + 6, 1, -2, 0, 2, 0, "double", "vertexdx");
    vertexy = D1(1, y_cells + 6, 0, -2, 0, 2, "double", "vertexy");
    vertexdy = D1(1, y_cells + 6, 0, -2, 0, 2, "double", "vertexdy");
    xx = D1(x_cells + 6, 1, -2, 0, 2, 0, "int", "xx");
    yy = D1(1, y_cells + 6, 0, -2, 0, 2, "int", "yy");

    S2D_00 = stencil(1, {0, 0}, "00");
    S2D_00_P10 = stencil(2, {0, 0, 1, 0}, "0,0:1,0");
    S2D_00_0P1 = stencil(2, {0, 0, 0, 1}, "0,0:0,1");
    S2D_00_M10 = stencil(2, {0, 0, -1, 0}, "0,0:-1,0");
    S2D_00_0M1 = stencil(2, {0, 0, 0, -1}, "0,0:0,-1");
    S2D_00_P10_M10 = stencil(3, {0, 0, 1, 0, -1, 0}, "0,0:1,0:-1,0");
    S2D_00_0P1_0M1 = stencil(3, {0, 0, 0, 1, 0, -1}, "0,0:0,1:0,-1");
    S2D_00_M10_M20 = stencil(3, {0, 0, -1, 0, -2, 0}, "0,0:-1,0:-2,0");
    S2D_00_0M1_0M2 = stencil(3, {0, 0, 0, -1, 0, -2}, "0,0:0,-1:0,-2");
    S2D_00_P20 = stencil(2, {0, 0, 2, 0}, "0,0:2,0");
    S2D_00_0P2 = stencil(2, {0, 0, 0, 2}, "0,0:0,2");
    S2D_00_M20 = stencil(2, {0, 0, -2, 0}, "0,0:-2,0");
    S2D_00_0M2 = stencil(2, {0, 0, 0, -2}, "0,0:0,-2");
    S2D_00_P30 = stencil(2, {0, 0, 3, 0}, "0,0:3,0");
    S2D_00_0P3 = stencil(2, {0, 0, 0, 3}, "0,0:0,3");
    S2D_00_M30 = stencil(2, {0, 0, -3, 0}, "0,0:-3,0");
    S2D_00_0M3 = stencil(2, {0, 0, 0, -3}, "0,0:0,-3");
    S2D_00_P40 = stencil(2, {0, 0, 4, 0}, "0,0:4,0");
    S2D_00_0P4 = stencil(2, {0, 0, 0, 4}, "0,0:0,4");
    S2D_00_M40 = stencil(2, {0, 0, -4, 0}, "0,0:-4,0");
    S2D_00_0M4 = stencil(2, {0, 0, 0, -4}, "0,0:0,-4");
    S2D_00_P10_0P1_P1P1 = stencil(4, {0, 0, 1, 0, 0, 1, 1, 1}, "0,0:1,0:0,1:1,1");
    S2D_00_M10_0M1_M1M1 = stencil(4, {0, 0, -1, 0, 0, -1, -1, -1}, "0,0:-1,0:0,-1:-1,-1");
    S2D_00_P10_0M1_P1M1 = stencil(4, {0, 0, 1, 0, 0, -1, 1, -1}, "0,0:1,0:0,-1:1,-1");
    S2D_00_0P1_M10_M1P1 = stencil(4, {0, 0, 0, 1, -1, 0, -1, 1}, "0,0:0,1:-1,0:-1,1");
    S2D_10_M10_01_0M1 = stencil(4, {1, 0, -1, 0, 0, 1, 0, -1}, "1,0:-1,0:0,1:0,-1");
    S2D_00_P10_M10_M20 = stencil(4, {0, 0, 1, 0, -1, 0, -2, 0}, "0,0:1,0:-1,0:-2,0");
    S2D_00_P10_M10_STRID2D_X = strided(3, {0, 0, 1, 0, -1, 0}, {1, 0}, "self_stride2D_x");
    S2D_00_0P1_0M1_0M2 = stencil(4, {0, 0, 0, 1, 0, -1, 0, -2}, "0,0:0,1:0,-1:0,-2");
    S2D_00_0P1_0M1_STRID2D_Y = strided(3, {0, 0, 0, 1, 0, -1}, {0, 1}, "self_stride2D_y");
    S2D_00_P10_P20_M10 = stencil(4, {0, 0, 1, 0, 2, 0, -1, 0}, "0,0:1,0:2,0:-1,0");
    S2D_00_0P1_0P2_0M1 = stencil(4, {0, 0, 0, 1, 0, 2, 0, -1}, "0,0:0,1:0,2:0,-1");
    S2D_00_STRID2D_X = strided(1, {0, 0}, {1, 0}, "s2D_00_stride2D_x");
    S2D_00_STRID2D_Y = strided(1, {0, 0}, {0, 1}, "s2D_00_stride2D_y");
    S2D_00_P10_STRID2D_X = strided(2, {0, 0, 1, 0}, {1, 0}, "s2D_00_P10_stride2D_x");
    S2D_00_0P1_STRID2D_Y = strided(2, {0, 0, 0, 1}, {0, 1}, "s2D_00_0P1_stride2D_y");
    S2D_00_M10_STRID2D_X = strided(2, {0, 0, -1, 0}, {1, 0}, "s2D_00_M10_stride2D_x");
    S2D_00_0M1_STRID2D_Y = strided(2, {0, 0, 0, -1}, {0, 1}, "s2D_00_0M1_stride2D_y");

    red_local_dt = r.decl_reduction(8, "double", "local_dt");
    red_xl_pos = r.decl_reduction(8, "double", "xl_pos");
    red_yl_pos = r.decl_reduction(8, "double", "yl_pos");
    red_vol = r.decl_reduction(8, "double", "vol");
    red_mass = r.decl_reduction(8, "double", "mass");
    red_ie = r.decl_reduction(8, "double", "ie");
    red_ke = r.decl_reduction(8, "double", "ke");
    red_press = r.decl_reduction(8, "double", "press");
    red_output = r.decl_reduction(12 * 8, "double", "output");
  }

  // initialise_chunk.cpp:40-95
  void initialise_chunk() {
    const int x_min = field.x_min, x_max = field.x_max, y_min = field.y_min, y_max = field.y_max;
    int rangex[] = {x_min - 2, x_max + 3, y_min - 2, y_min - 1};
    int rangey[] = {x_min - 2, x_min - 1, y_min - 2, y_max + 3};
    int rangefull[] = {-2, grid.x_cells + 8, -2, grid.y_cells + 8};
    loop("initialise_chunk_kernel_xx", "initialise_chunk_kernel_xx", rangefull,
         {dat(xx, S2D_00_STRID2D_X, ACC_WRITE), arg_idx()});
    loop("initialise_chunk_kernel_yy", "initialise_chunk_kernel_yy", rangefull,
         {dat(yy, S2D_00_STRID2D_Y, ACC_WRITE), arg_idx()});
    loop("initialise_chunk_kernel_x", "initialise_chunk_kernel_x", rangex,
         {dat(vertexx, S2D_00_STRID2D_X, ACC_WRITE), dat(xx, S2D_00_STRID2D_X, ACC_READ),
          dat(vertexdx, S2D_00_STRID2D_X, ACC_WRITE)});
    loop("initialise_chunk_kernel_y", "initialise_chunk_kernel_y", rangey,
         {dat(vertexy, S2D_00_STRID2D_Y, ACC_WRITE), dat(yy, S2D_00_STRID2D_Y, ACC_READ),
          dat(vertexdy, S2D_00_STRID2D_Y, ACC_WRITE)});
    rangex[0] = x_min - 2; rangex[1] = x_max + 2; rangex[2] = y_min - 2; rangex[3] = y_min - 1;
    loop("initialise_chunk_kernel_cellx", "initialise_chunk_kernel_cellx", rangex,
         {dat(vertexx, S2D_00_P10_STRID2D_X, ACC_READ), dat(cellx, S2D_00_STRID2D_X, ACC_WRITE),
          dat(celldx, S2D_00_STRID2D_X, ACC_WRITE)});
    rangey[0] = x_min - 2; rangey[1] = x_min - 1; rangey[2] = y_min - 2; rangey[3] = y_max + 2;
    loop("initialise_chunk_kernel_celly", "initialise_chunk_kernel_celly", rangey,
         {dat(vertexy, S2D_00_0P1_STRID2D_Y, ACC_READ), dat(celly, S2D_00_STRID2D_Y, ACC_WRITE),
          dat(celldy, S2D_00_STRID2D_Y, ACC_WRITE)});
    int rangexy[] = {x_min - 2, x_max + 2, y_min - 2, y_max + 2};
    loop("initialise_chunk_kernel_volume", "initialise_chunk_kernel_volume", rangexy,
         {dat(volume, S2D_00, ACC_WRITE), dat(celldy, S2D_00_STRID2D_Y, ACC_READ), dat(xarea, S2D_00, ACC_WRITE),
          dat(celldx, S2D_00_STRID2D_X, ACC_READ), dat(yarea, S2D_00, ACC_WRITE)});
  }

  // generate.cpp:39-58
  void generate() {
    int rangexy[] = {field.x_min - 2, field.x_max + 2, field.y_min - 2, field.y_max + 2};
    loop("generate_chunk_kernel", "generate_chunk_kernel", rangexy,
         {dat(vertexx, S2D_00_P10_M10_STRID2D_X, ACC_READ), dat(vertexy, S2D_00_0P1_0M1_STRID2D_Y, ACC_READ),
          dat(energy0, S2D_00, ACC_WRITE), dat(density0, S2D_00, ACC_WRITE), dat(xvel0, S2D_00, ACC_WRITE),
          dat(yvel0, S2D_00, ACC_WRITE), dat(cellx, S2D_00_P10_M10_STRID2D_X, ACC_READ),
          dat(celly, S2D_00_0P1_0M1_STRID2D_Y, ACC_READ)});
  }

  // ideal_gas.cpp:38-63
  void ideal_gas(int predict) {
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    int d = predict ? density1 : density0, e = predict ? energy1 : energy0;
    loop("ideal_gas_kernel", "ideal_gas_kernel", rng,
         {dat(d, S2D_00, ACC_READ), dat(e, S2D_00, ACC_READ), dat(pressure, S2D_00, ACC_WRITE),
          dat(soundspeed, S2D_00, ACC_WRITE)});
  }

  // update_halo.cpp:40-386
  void update_halo(const int *f, int depth) {
    const int x_min = field.x_min, x_max = field.x_max, y_min = field.y_min, y_max = field.y_max;
    Arg gbl = arg_gbl(f, NUM_FIELDS, 4, ACC_READ);
    if (f[FIELD_DENSITY0] || f[FIELD_DENSITY1] || f[FIELD_ENERGY0] || f[FIELD_ENERGY1] || f[FIELD_PRESSURE] ||
        f[FIELD_VISCOSITY] || f[FIELD_SOUNDSPEED]) {
      auto k1 = [&](const char *k, const char *nm, const int *rng, int st) {
        loop(k, nm, rng,
             {dat_opt(density0, st, ACC_RW, f[FIELD_DENSITY0]), dat_opt(density1, st, ACC_RW, f[FIELD_DENSITY1]),
              dat_opt(energy0, st, ACC_RW, f[FIELD_ENERGY0]), dat_opt(energy1, st, ACC_RW, f[FIELD_ENERGY1]),
              dat_opt(pressure, st, ACC_RW, f[FIELD_PRESSURE]), dat_opt(viscosity, st, ACC_RW, f[FIELD_VISCOSITY]),
              dat_opt(soundspeed, st, ACC_RW, f[FIELD_SOUNDSPEED]), gbl});
      };
      int b2[] = {x_min - depth, x_max + depth, y_min - 2, y_min - 1};
      if (depth == 2) k1("update_halo_kernel1_b2", "update_halo_kernel1", b2, S2D_00_0P3);
      int b1[] = {x_min - depth, x_max + depth, y_min - 1, y_min};
      k1("update_halo_kernel1_b1", "update_halo_kernel1", b1, S2D_00_0P1);
      int t2[] = {x_min - depth, x_max + depth, y_max + 1, y_max + 2};
      if (depth == 2) k1("update_halo_kernel1_t2", "update_halo_kernel1", t2, S2D_00_0M3);
      int t1[] = {x_min - depth, x_max + depth, y_max, y_max + 1};
      k1("update_halo_kernel1_t1", "update_halo_kernel1", t1, S2D_00_0M1);
      int l2[] = {x_min - 2, x_min - 1, y_min - depth, y_max + depth};
      if (depth == 2) k1("update_halo_kernel1_l2", "update_halo_kernel", l2, S2D_00_P30);
      int l1[] = {x_min - 1, x_min, y_min - depth, y_max + depth};
      k1("update_halo_kernel1_l1", "update_halo_kernel", l1, S2D_00_P10);
      int r2[] = {x_max + 1, x_max + 2, y_min - depth, y_max + depth};
      if (depth == 2) k1("update_halo_kernel1_r2", "update_halo_kernel", r2, S2D_00_M30);
      int r1[] = {x_max, x_max + 1, y_min - depth, y_max + depth};
      k1("update_halo_kernel1_r1", "update_halo_kernel", r1, S2D_00_M10);
    }
    auto k2 = [&](const char *k, const int *rng, int a, int fa, int b, int fb, int st) {
      loop(k, k, rng, {dat_opt(a, st, ACC_RW, f[fa]), dat_opt(b, st, ACC_RW, f[fb]), gbl});
    };
    if (f[FIELD_XVEL0] || f[FIELD_XVEL1]) {
      const int a = xvel0, b = xvel1, fa = FIELD_XVEL0, fb = FIELD_XVEL1;
      int b2[] = {x_min - depth, x_max + 1 + depth, y_min - 2, y_min - 1};
      if (depth == 2) k2("update_halo_kernel2_xvel_plus_4_a", b2, a, fa, b, fb, S2D_00_0P4);
      int b1[] = {x_min - depth, x_max + 1 + depth, y_min - 1, y_min};
      k2("update_halo_kernel2_xvel_plus_2_a", b1, a, fa, b, fb, S2D_00_0P2);
      int t2[] = {x_min - depth, x_max + 1 + depth, y_max + 2, y_max + 3};
      if (depth == 2) k2("update_halo_kernel2_xvel_plus_4_b", t2, a, fa, b, fb, S2D_00_0M4);
      int t1[] = {x_min - depth, x_max + 1 + depth, y_max + 1, y_max + 2};
      k2("update_halo_kernel2_xvel_plus_2_b", t1, a, fa, b, fb, S2D_00_0M2);
      int l2[] = {x_min - 2, x_min - 1, y_min - depth, y_max + 1 + depth};
      if (depth == 2) k2("update_halo_kernel2_xvel_minus_4_a", l2, a, fa, b, fb, S2D_00_P40);
      int l1[] = {x_min - 1, x_min, y_min - depth, y_max + 1 + depth};
      k2("update_halo_kernel2_xvel_minus_2_a", l1, a, fa, b, fb, S2D_00_P20);
      int r2[] = {x_max + 2, x_max + 3, y_min - depth, y_max + 1 + depth};
      if (depth == 2) k2("update_halo_kernel2_xvel_minus_4_b", r2, a, fa, b, fb, S2D_00_M40);
      int r1[] = {x_max + 1, x_max + 2, y_min - depth, y_max + 1 + depth};
      k2("update_halo_kernel2_xvel_minus_2_b", r1, a, fa, b, fb, S2D_00_M20);
    }
    if (f[FIELD_YVEL0] || f[FIELD_YVEL1]) {
      const int a = yvel0, b = yvel1, fa = FIELD_YVEL0, fb = FIELD_YVEL1;
      int b2[] = {x_min - depth, x_max + 1 + depth, y_min - 2, y_min - 1};
      if (depth == 2) k2("update_halo_kernel2_yvel_minus_4_a", b2, a, fa, b, fb, S2D_00_0P4);
      int b1[] = {x_min - depth, x_max + 1 + depth, y_min - 1, y_min};
      k2("update_halo_kernel2_yvel_minus_2_a", b1, a, fa, b, fb, S2D_00_0P2);
      int t2[] = {x_min - depth, x_max + 1 + depth, y_max + 2, y_max + 3};
      if (depth == 2) k2("update_halo_kernel2_yvel_minus_4_b", t2, a, fa, b, fb, S2D_00_0M4);
      int t1[] = {x_min - depth, x_max + 1 + depth, y_max + 1, y_max + 2};
      k2("update_halo_kernel2_yvel_minus_2_b", t1, a, fa, b, fb, S2D_00_0M2);
      int l2[] = {x_min - 2, x_min - 1, y_min - depth, y_max + 1 + depth};
      if (depth == 2) k2("update_halo_kernel2_yvel_plus_4_a", l2, a, fa, b, fb, S2D_00_P40);
      int l1[] = {x_min - 1, x_min, y_min - depth, y_max + 1 + depth};
      k2("update_halo_kernel2_yvel_plus_2_a", l1, a, fa, b, fb, S2D_00_P20);
      int r2[] = {x_max + 2, x_max + 3, y_min - depth, y_max + 1 + depth};
      if (depth == 2) k2("update_halo_kernel2_yvel_plus_4_b", r2, a, fa, b, fb, S2D_00_M40);
      int r1[] = {x_max + 1, x_max + 2, y_min - depth, y_max + 1 + depth};
      k2("update_halo_kernel2_yvel_plus_2_b", r1, a, fa, b, fb, S2D_00_M20);
    }
    if (f[FIELD_MASS_FLUX_X] || f[FIELD_VOL_FLUX_X]) {
      const int a = vol_flux_x, b = mass_flux_x, fa = FIELD_VOL_FLUX_X, fb = FIELD_MASS_FLUX_X;
      int b2[] = {x_min - depth, x_max + 1 + depth, y_min - 2, y_min - 1};
      if (depth == 2) k2("update_halo_kernel3_plus_4_a", b2, a, fa, b, fb, S2D_00_0P4);
      int b1[] = {x_min - depth, x_max + 1 + depth, y_min - 1, y_min};
      k2("update_halo_kernel3_plus_2_a", b1, a, fa, b, fb, S2D_00_0P2);
      int t2[] = {x_min - depth, x_max + 1 + depth, y_max + 1, y_max + 2};
      if (depth == 2) k2("update_halo_kernel3_plus_4_b", t2, a, fa, b, fb, S2D_00_0M4);
      int t1[] = {x_min - depth, x_max + 1 + depth, y_max, y_max + 1};
      k2("update_halo_kernel3_plus_2_b", t1, a, fa, b, fb, S2D_00_0M2);
      int l2[] = {x_min - 2, x_min - 1, y_min - depth, y_max + depth};
      if (depth == 2) k2("update_halo_kernel3_minus_4_a", l2, a, fa, b, fb, S2D_00_P40);
      int l1[] = {x_min - 1, x_min, y_min - depth, y_max + depth};
      k2("update_halo_kernel3_minus_2_a", l1, a, fa, b, fb, S2D_00_P20);
      int r2[] = {x_max + 2, x_max + 3, y_min - depth, y_max + depth};
      if (depth == 2) k2("update_halo_kernel3_minus_4_b", r2, a, fa, b, fb, S2D_00_M40);
      int r1[] = {x_max + 1, x_max + 2, y_min - depth, y_max + depth};
      k2("update_halo_kernel3_minus_2_b", r1, a, fa, b, fb, S2D_00_M20);
    }
    if (f[FIELD_MASS_FLUX_Y] || f[FIELD_VOL_FLUX_Y]) {
      const int a = vol_flux_y, b = mass_flux_y, fa = FIELD_VOL_FLUX_Y, fb = FIELD_MASS_FLUX_Y;
      int b2[] = {x_min - depth, x_max + depth, y_min - 2, y_min - 1};
      if (depth == 2) k2("update_halo_kernel4_minus_4_a", b2, a, fa, b, fb, S2D_00_0P4);
      int b1[] = {x_min - depth, x_max + depth, y_min - 1, y_min};
      k2("update_halo_kernel4_minus_2_a", b1, a, fa, b, fb, S2D_00_0P2);
      int t2[] = {x_min - depth, x_max + depth, y_max + 2, y_max + 3};
      if (depth == 2) k2("update_halo_kernel4_minus_4_b", t2, a, fa, b, fb, S2D_00_0M4);
      int t1[] = {x_min - depth, x_max + depth, y_max + 1, y_max + 2};
      k2("update_halo_kernel4_minus_2_b", t1, a, fa, b, fb, S2D_00_0M2);
      int l2[] = {x_min - 2, x_min - 1, y_min - depth, y_max + 1 + depth};
      if (depth == 2) k2("update_halo_kernel4_plus_4_a", l2, a, fa, b, fb, S2D_00_P40);
      int l1[] = {x_min - 1, x_min, y_min - depth, y_max + 1 + depth};
      k2("update_halo_kernel4_plus_2_a", l1, a, fa, b, fb, S2D_00_P20);
      int r2[] = {x_max + 1, x_max + 2, y_min - depth, y_max + 1 + depth};
      if (depth == 2) k2("update_halo_kernel4_plus_4_b", r2, a, fa, b, fb, S2D_00_M40);
      int r1[] = {x_max, x_max + 1, y_min - depth, y_max + 1 + depth};
      k2("update_halo_kernel4_plus_2_b", r1, a, fa, b, fb, S2D_00_M20);
    }
  }

  void set_fields(std::initializer_list<int> on) {
    for (int i = 0; i < NUM_FIELDS; i++) fields[i] = 0;
    for (int i : on) fields[i] = 1;
  }

  // field_summary.cpp:44-110
  void field_summary() {
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    ideal_gas(0);
    loop("field_summary_kernel", "field_summary_kernel", rng,
         {dat(volume, S2D_00, ACC_READ), dat(density0, S2D_00, ACC_READ), dat(energy0, S2D_00, ACC_READ),
          dat(pressure, S2D_00, ACC_READ), dat(xvel0, S2D_00_P10_0P1_P1P1, ACC_READ),
          dat(yvel0, S2D_00_P10_0P1_P1P1, ACC_READ), arg_reduce(red_vol, 1, ACC_INC),
          arg_reduce(red_mass, 1, ACC_INC), arg_reduce(red_ie, 1, ACC_INC), arg_reduce(red_ke, 1, ACC_INC),
          arg_reduce(red_press, 1, ACC_INC)});
    double vol = 0, mass = 0, ie = 0, ke = 0, press = 0;
    r.reduction_result(red_vol, &vol);
    r.reduction_result(red_mass, &mass);
    r.reduction_result(red_ie, &ie);
    r.reduction_result(red_ke, &ke);
    r.reduction_result(red_press, &press);
    double row[8] = {(double)step, clover_time, vol, mass, ie, ke, press, dt};
    summaries.insert(summaries.end(), row, row + 8);
  }

  void viscosity_func() {  // viscosity.cpp:41-58
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("viscosity_kernel", "viscosity_kernel", rng,
         {dat(xvel0, S2D_00_P10_0P1_P1P1, ACC_READ), dat(yvel0, S2D_00_P10_0P1_P1P1, ACC_READ),
          dat(celldx, S2D_00_P10_STRID2D_X, ACC_READ), dat(celldy, S2D_00_0P1_STRID2D_Y, ACC_READ),
          dat(pressure, S2D_10_M10_01_0M1, ACC_READ), dat(density0, S2D_00, ACC_READ),
          dat(viscosity, S2D_00, ACC_WRITE)});
  }

  // calc_dt.cpp:37-131
  void calc_dt(double *local_dt, double *xl_pos, double *yl_pos, int *jldt, int *kldt) {
    double jk_control = 1.1;
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("calc_dt_kernel", "calc_dt_kernel", rng,
         {dat(celldx, S2D_00_P10_STRID2D_X, ACC_READ), dat(celldy, S2D_00_0P1_STRID2D_Y, ACC_READ),
          dat(soundspeed, S2D_00, ACC_READ), dat(viscosity, S2D_00, ACC_READ), dat(density0, S2D_00, ACC_READ),
          dat(xvel0, S2D_00_P10_0P1_P1P1, ACC_READ), dat(xarea, S2D_00_P10, ACC_READ),
          dat(volume, S2D_00, ACC_READ), dat(yvel0, S2D_00_P10_0P1_P1P1, ACC_READ),
          dat(yarea, S2D_00_0P1, ACC_READ), dat(work_array1, S2D_00, ACC_WRITE)});
    loop("calc_dt_kernel_min", "calc_dt_kernel_min", rng,
         {dat(work_array1, S2D_00, ACC_READ), arg_reduce(red_local_dt, 1, ACC_MIN)});
    jk_control = jk_control - (jk_control - (int)(jk_control));
    *jldt = ((int)jk_control) % (field.x_max - 2);
    *kldt = 1 + (jk_control / (field.x_max - 2));
    int getpoint[] = {*jldt - 1 + 2, *jldt + 2, *kldt - 1 + 2, *kldt + 2};
    loop("calc_dt_kernel_get", "calc_dt_kernel_getx", getpoint,
         {dat(cellx, S2D_00_STRID2D_X, ACC_READ), dat(celly, S2D_00_STRID2D_Y, ACC_READ),
          arg_reduce(red_xl_pos, 1, ACC_INC), arg_reduce(red_yl_pos, 1, ACC_INC)});
    r.reduction_result(red_local_dt, local_dt);
    r.reduction_result(red_xl_pos, xl_pos);
    r.reduction_result(red_yl_pos, yl_pos);
    *local_dt = op_min(*local_dt, g_big);
    if (*local_dt < dtmin) throw Error(E_STATE, "cloverleaf: timestep below dtmin (calc_dt.cpp:99-125)");
  }

  // time_step.cpp:39-130
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
    r.decl_const("cloverleaf/dt", 1, "double", &dt_temp);
    dt = dt_temp;
    if (dt < dtmin) throw Error(E_STATE, "cloverleaf: small timestep (time_step.cpp:123-126)");
    dtold = dt;
  }

  void revert() {  // revert.cpp:39-57
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("revert_kernel", "revert_kernel", rng,
         {dat(density0, S2D_00, ACC_READ), dat(density1, S2D_00, ACC_WRITE), dat(energy0, S2D_00, ACC_READ),
          dat(energy1, S2D_00, ACC_WRITE)});
  }

  // PdV.cpp:41-117
  void PdV(int predict) {
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    if (predict) {
      loop("PdV_kernel_predict", "PdV_kernel_predict", rng,
           {dat(xarea, S2D_00_P10_0P1_P1P1, ACC_READ), dat(xvel0, S2D_00_P10_0P1_P1P1, ACC_READ),
            dat(yarea, S2D_00_P10_0P1_P1P1, ACC_READ), dat(yvel0, S2D_00_P10_0P1_P1P1, ACC_READ),
            dat(work_array1, S2D_00, ACC_WRITE), dat(volume, S2D_00, ACC_READ), dat(pressure, S2D_00, ACC_READ),
            dat(density0, S2D_00, ACC_READ), dat(density1, S2D_00, ACC_WRITE), dat(viscosity, S2D_00, ACC_READ),
            dat(energy0, S2D_00, ACC_READ), dat(energy1, S2D_00, ACC_WRITE)});
    } else {
      loop("PdV_kernel_nopredict", "PdV_kernel_nopredict", rng,
           {dat(xarea, S2D_00_P10_0P1_P1P1, ACC_READ), dat(xvel0, S2D_00_P10_0P1_P1P1, ACC_READ),
            dat(xvel1, S2D_00_P10_0P1_P1P1, ACC_READ), dat(yarea, S2D_00_P10_0P1_P1P1, ACC_READ),
            dat(yvel0, S2D_00_P10_0P1_P1P1, ACC_READ), dat(yvel1, S2D_00_P10_0P1_P1P1, ACC_READ),
            dat(work_array1, S2D_00, ACC_WRITE), dat(volume, S2D_00, ACC_READ), dat(pressure, S2D_00, ACC_READ),
            dat(density0, S2D_00, ACC_READ), dat(density1, S2D_00, ACC_WRITE), dat(viscosity, S2D_00, ACC_READ),
            dat(energy0, S2D_00, ACC_READ), dat(energy1, S2D_00, ACC_WRITE)});
    }
    if (predict) {
      ideal_gas(1);
      set_fields({FIELD_PRESSURE});
      update_halo(fields, 1);
      revert();
    }
  }

  void accelerate() {  // accelerate.cpp:39-63
    int rng[] = {field.x_min, field.x_max + 1, field.y_min, field.y_max + 1};
    loop("accelerate_kernel", "accelerate_kernel", rng,
         {dat(density0, S2D_00_M10_0M1_M1M1, ACC_READ), dat(volume, S2D_00_M10_0M1_M1M1, ACC_READ),
          dat(work_array1, S2D_00, ACC_WRITE), dat(xvel0, S2D_00, ACC_READ), dat(xvel1, S2D_00, ACC_WRITE),
          dat(xarea, S2D_00_0M1, ACC_READ), dat(pressure, S2D_00_M10_0M1_M1M1, ACC_READ),
          dat(yvel0, S2D_00, ACC_READ), dat(yvel1, S2D_00, ACC_WRITE), dat(yarea, S2D_00_M10, ACC_READ),
          dat(viscosity, S2D_00_M10_0M1_M1M1, ACC_READ)});
  }

  void flux_calc() {  // flux_calc.cpp:38-64
    int rx[] = {field.x_min, field.x_max + 1, field.y_min, field.y_max};
    loop("flux_calc_kernelx", "flux_calc_kernelx", rx,
         {dat(vol_flux_x, S2D_00, ACC_WRITE), dat(xarea, S2D_00, ACC_READ), dat(xvel0, S2D_00_0P1, ACC_READ),
          dat(xvel1, S2D_00_0P1, ACC_READ)});
    int ry[] = {field.x_min, field.x_max, field.y_min, field.y_max + 1};
    loop("flux_calc_kernely", "flux_calc_kernely", ry,
         {dat(vol_flux_y, S2D_00, ACC_WRITE), dat(yarea, S2D_00, ACC_READ), dat(yvel0, S2D_00_P10, ACC_READ),
          dat(yvel1, S2D_00_P10, ACC_READ)});
  }

  // advec_cell.cpp:38-147
  void advec_cell(int sweep_number, int dir) {
    const int x_min = field.x_min, x_max = field.x_max, y_min = field.y_min, y_max = field.y_max;
    int rangexy[] = {x_min - 2, x_max + 2, y_min - 2, y_max + 2};
    int inner[] = {x_min, x_max, y_min, y_max};
    int plus2x[] = {x_min, x_max + 2, y_min, y_max};
    int plus2y[] = {x_min, x_max, y_min, y_max + 2};
    if (dir == 1) {
      if (sweep_number == 1)
        loop("advec_cell_kernel1_xdir", "advec_cell_kernel1_xdir", rangexy,
             {dat(work_array1, S2D_00, ACC_WRITE), dat(work_array2, S2D_00, ACC_WRITE), dat(volume, S2D_00, ACC_READ),
              dat(vol_flux_x, S2D_00_P10, ACC_READ), dat(vol_flux_y, S2D_00_0P1, ACC_READ)});
      else
        loop("advec_cell_kernel2_xdir", "advec_cell_kernel2_xdir", rangexy,
             {dat(work_array1, S2D_00, ACC_WRITE), dat(work_array2, S2D_00, ACC_WRITE), dat(volume, S2D_00, ACC_READ),
              dat(vol_flux_x, S2D_00_P10, ACC_READ)});
      loop("advec_cell_kernel3_xdir", "advec_cell_kernel3_xdir", plus2x,
           {dat(vol_flux_x, S2D_00, ACC_READ), dat(work_array1, S2D_00_M10, ACC_READ),
            dat(xx, S2D_00_P10_STRID2D_X, ACC_READ), dat(vertexdx, S2D_00_P10_M10_STRID2D_X, ACC_READ),
            dat(density1, S2D_00_P10_M10_M20, ACC_READ), dat(energy1, S2D_00_P10_M10_M20, ACC_READ),
            dat(mass_flux_x, S2D_00, ACC_WRITE), dat(work_array7, S2D_00, ACC_WRITE)});
      loop("advec_cell_kernel4_xdir", "advec_cell_kernel4_xdir", inner,
           {dat(density1, S2D_00, ACC_RW), dat(energy1, S2D_00, ACC_RW), dat(mass_flux_x, S2D_00_P10, ACC_READ),
            dat(vol_flux_x, S2D_00_P10, ACC_READ), dat(work_array1, S2D_00, ACC_READ),
            dat(work_array2, S2D_00, ACC_READ), dat(work_array3, S2D_00, ACC_WRITE),
            dat(work_array4, S2D_00, ACC_WRITE), dat(work_array5, S2D_00, ACC_WRITE),
            dat(work_array6, S2D_00, ACC_WRITE), dat(work_array7, S2D_00_P10, ACC_READ)});
    } else {
      if (sweep_number == 1)
        loop("advec_cell_kernel1_ydir", "advec_cell_kernel1_ydir", rangexy,
             {dat(work_array1, S2D_00, ACC_WRITE), dat(work_array2, S2D_00, ACC_WRITE), dat(volume, S2D_00, ACC_READ),
              dat(vol_flux_x, S2D_00_P10, ACC_READ), dat(vol_flux_y, S2D_00_0P1, ACC_READ)});
      else
        loop("advec_cell_kernel2_ydir", "advec_cell_kernel2_ydir", rangexy,
             {dat(work_array1, S2D_00, ACC_WRITE), dat(work_array2, S2D_00, ACC_WRITE), dat(volume, S2D_00, ACC_READ),
              dat(vol_flux_y, S2D_00_0P1, ACC_READ)});
      loop("advec_cell_kernel3_ydir", "advec_cell_kernel3_ydir", plus2y,
           {dat(vol_flux_y, S2D_00, ACC_READ), dat(work_array1, S2D_00_0M1, ACC_READ),
            dat(yy, S2D_00_0P1_STRID2D_Y, ACC_READ), dat(vertexdy, S2D_00_0P1_0M1_STRID2D_Y, ACC_READ),
            dat(density1, S2D_00_0P1_0M1_0M2, ACC_READ), dat(energy1, S2D_00_0P1_0M1_0M2, ACC_READ),
            dat(mass_flux_y, S2D_00, ACC_WRITE), dat(work_array7, S2D_00, ACC_WRITE)});
      loop("advec_cell_kernel4_ydir", "advec_cell_kernel4_ydir", inner,
           {dat(density1, S2D_00, ACC_RW), dat(energy1, S2D_00, ACC_RW), dat(mass_flux_y, S2D_00_0P1, ACC_READ),
            dat(vol_flux_y, S2D_00_0P1, ACC_READ), dat(work_array1, S2D_00, ACC_READ),
            dat(work_array2, S2D_00, ACC_READ), dat(work_array3, S2D_00, ACC_WRITE),
            dat(work_array4, S2D_00, ACC_WRITE), dat(work_array5, S2D_00, ACC_WRITE),
            dat(work_array6, S2D_00, ACC_WRITE), dat(work_array7, S2D_00_0P1, ACC_READ)});
    }
  }

  // advec_mom.cpp:40-163
  void advec_mom(int which_vel, int sweep_number, int dir) {
    const int x_min = field.x_min, x_max = field.x_max, y_min = field.y_min, y_max = field.y_max;
    int rangexy[] = {x_min - 2, x_max + 2, y_min - 2, y_max + 2};
    int vel1 = which_vel == 1 ? xvel1 : yvel1;
    int mom_sweep = dir + 2 * (sweep_number - 1);
    if (mom_sweep == 1)
      loop("advec_mom_kernel_x1", "advec_mom_kernel_x1", rangexy,
           {dat(work_array6, S2D_00, ACC_WRITE), dat(work_array7, S2D_00, ACC_WRITE), dat(volume, S2D_00, ACC_READ),
            dat(vol_flux_x, S2D_00_P10, ACC_READ), dat(vol_flux_y, S2D_00_0P1, ACC_READ)});
    else if (mom_sweep == 2)
      loop("advec_mom_kernel_y1", "advec_mom_kernel_y1", rangexy,
           {dat(work_array6, S2D_00, ACC_WRITE), dat(work_array7, S2D_00, ACC_WRITE), dat(volume, S2D_00, ACC_READ),
            dat(vol_flux_x, S2D_00_P10, ACC_READ), dat(vol_flux_y, S2D_00_0P1, ACC_READ)});
    else if (mom_sweep == 3)
      loop("advec_mom_kernel_x2", "advec_mom_kernel_x2", rangexy,
           {dat(work_array6, S2D_00, ACC_WRITE), dat(work_array7, S2D_00, ACC_WRITE), dat(volume, S2D_00, ACC_READ),
            dat(vol_flux_y, S2D_00_0P1, ACC_READ)});
    else if (mom_sweep == 4)
      loop("advec_mom_kernel_y2", "advec_mom_kernel_y2", rangexy,
           {dat(work_array6, S2D_00, ACC_WRITE), dat(work_array7, S2D_00, ACC_WRITE), dat(volume, S2D_00, ACC_READ),
            dat(vol_flux_x, S2D_00_P10, ACC_READ)});
    int fullx_party_1[] = {x_min - 2, x_max + 2, y_min, y_max + 1};
    int partx_party_1[] = {x_min - 1, x_max + 2, y_min, y_max + 1};
    int fully_party_1[] = {x_min, x_max + 1, y_min - 2, y_max + 2};
    int partx_party_2[] = {x_min, x_max + 1, y_min - 1, y_max + 2};
    int inner_plus1[] = {x_min, x_max + 1, y_min, y_max + 1};
    if (dir == 1) {
      loop("advec_mom_kernel_mass_flux_x", "advec_mom_kernel_mass_flux_x", fullx_party_1,
           {dat(work_array1, S2D_00, ACC_WRITE), dat(mass_flux_x, S2D_00_P10_0M1_P1M1, ACC_READ)});
      loop("advec_mom_kernel_post_pre_advec_x", "advec_mom_kernel_post_pre_advec_x", partx_party_1,
           {dat(work_array2, S2D_00, ACC_WRITE), dat(work_array7, S2D_00_M10_0M1_M1M1, ACC_READ),
            dat(density1, S2D_00_M10_0M1_M1M1, ACC_READ), dat(work_array3, S2D_00, ACC_WRITE),
            dat(work_array1, S2D_00_M10, ACC_READ)});
      int r1[] = {x_min - 1, x_max + 1, y_min, y_max + 1};
      loop("advec_mom_kernel1_x_nonvector", "advec_mom_kernel1_x", r1,
           {dat(work_array1, S2D_00, ACC_READ), dat(work_array3, S2D_00_P10, ACC_READ),
            dat(work_array5, S2D_00, ACC_WRITE), dat(celldx, S2D_00_P10_M10_STRID2D_X, ACC_READ),
            dat(vel1, S2D_00_P10_P20_M10, ACC_READ)});
      loop("advec_mom_kernel2_x", "advec_mom_kernel2_x", inner_plus1,
           {dat(vel1, S2D_00, ACC_RW), dat(work_array2, S2D_00, ACC_READ), dat(work_array3, S2D_00, ACC_READ),
            dat(work_array5, S2D_00_M10, ACC_READ)});
    } else if (dir == 2) {
      loop("advec_mom_kernel_mass_flux_y", "advec_mom_kernel_mass_flux_y", fully_party_1,
           {dat(work_array1, S2D_00, ACC_WRITE), dat(mass_flux_y, S2D_00_0P1_M10_M1P1, ACC_READ)});
      loop("advec_mom_kernel_post_pre_advec_y", "advec_mom_kernel_post_pre_advec_y", partx_party_2,
           {dat(work_array2, S2D_00, ACC_WRITE), dat(work_array7, S2D_00_M10_0M1_M1M1, ACC_READ),
            dat(density1, S2D_00_M10_0M1_M1M1, ACC_READ), dat(work_array3, S2D_00, ACC_WRITE),
            dat(work_array1, S2D_00_0M1, ACC_READ)});
      int r1[] = {x_min, x_max + 1, y_min - 1, y_max + 1};
      loop("advec_mom_kernel1_y_nonvector", "advec_mom_kernel1_y", r1,
           {dat(work_array1, S2D_00, ACC_READ), dat(work_array3, S2D_00_0P1, ACC_READ),
            dat(work_array5, S2D_00, ACC_WRITE), dat(celldy, S2D_00_0P1_0M1_STRID2D_Y, ACC_READ),
            dat(vel1, S2D_00_0P1_0P2_0M1, ACC_READ)});
      loop("advec_mom_kernel2_y", "advec_mom_kernel2_y", inner_plus1,
           {dat(vel1, S2D_00, ACC_RW), dat(work_array2, S2D_00, ACC_READ), dat(work_array3, S2D_00, ACC_READ),
            dat(work_array5, S2D_00_0M1, ACC_READ)});
    }
  }

  // advection.cpp:38-121
  void advection() {
    const int g_xdir = 1, g_ydir = 2;
    int sweep_number = 1;
    int direction = advect_x ? g_xdir : g_ydir;
    set_fields({FIELD_DENSITY1, FIELD_ENERGY1, FIELD_VOL_FLUX_X, FIELD_VOL_FLUX_Y});
    update_halo(fields, 2);
    advec_cell(sweep_number, direction);
    if (direction == g_xdir)
      set_fields({FIELD_DENSITY1, FIELD_ENERGY1, FIELD_XVEL1, FIELD_YVEL1, FIELD_MASS_FLUX_X});
    else
      set_fields({FIELD_DENSITY1, FIELD_ENERGY1, FIELD_XVEL1, FIELD_YVEL1, FIELD_MASS_FLUX_Y});
    update_halo(fields, 2);
    advec_mom(g_xdir, sweep_number, direction);
    advec_mom(g_ydir, sweep_number, direction);
    sweep_number = 2;
    direction = advect_x ? g_ydir : g_xdir;
    advec_cell(sweep_number, direction);
    set_fields({FIELD_DENSITY1, FIELD_ENERGY1, FIELD_XVEL1, FIELD_YVEL1, FIELD_MASS_FLUX_X, FIELD_MASS_FLUX_Y});
    update_halo(fields, 2);
    advec_mom(g_xdir, sweep_number, direction);
    advec_mom(g_ydir, sweep_number, direction);
  }

  void reset_field() {  // reset_field.cpp:39-64
    int inner[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("reset_field_kernel1", "reset_field_kernel1", inner,
         {dat(density0, S2D_00, ACC_WRITE), dat(density1, S2D_00, ACC_READ), dat(energy0, S2D_00, ACC_WRITE),
          dat(energy1, S2D_00, ACC_READ)});
    int plus1[] = {field.x_min, field.x_max + 1, field.y_min, field.y_max + 1};
    loop("reset_field_kernel2", "reset_field_kernel2", plus1,
         {dat(xvel0, S2D_00, ACC_WRITE), dat(xvel1, S2D_00, ACC_READ), dat(yvel0, S2D_00, ACC_WRITE),
          dat(yvel1, S2D_00, ACC_READ)});
  }

  // clover_leaf.cpp:133-160 + start.cpp:44-112
  void setup(const ops_b200_clover_deck &deck) {
    read_input(deck);
    r.decl_const("cloverleaf/g_small", 1, "double", &g_small);
    r.decl_const("cloverleaf/g_big", 1, "double", &g_big);
    r.decl_const("cloverleaf/dtc_safe", 1, "double", &dtc_safe);
    r.decl_const("cloverleaf/dtu_safe", 1, "double", &dtu_safe);
    r.decl_const("cloverleaf/dtv_safe", 1, "double", &dtv_safe);
    r.decl_const("cloverleaf/dtdiv_safe", 1, "double", &dtdiv_safe);
    r.decl_const("cloverleaf/field", 1, "field_type", &field);
    r.decl_const("cloverleaf/grid", 1, "grid_type", &grid);
    r.decl_const("cloverleaf/number_of_states", 1, "int", &number_of_states);
    r.decl_const("cloverleaf/states", number_of_states, "state_type", states);
    r.decl_const("cloverleaf/g_circ", 1, "int", &g_circ);
    r.decl_const("cloverleaf/g_point", 1, "int", &g_point);
    r.decl_const("cloverleaf/g_rect", 1, "int", &g_rect);
    r.decl_const("cloverleaf/dt", 1, "double", &dt);
    clover_time = 0.0;
    step = 0;
    dtold = dtinit;
    dt = dtinit;
    build_field();
    r.partition("2D_BLOCK_DECOMPSE");  // build_field.cpp:235
    initialise_chunk();
    generate();
    advect_x = 1;
    ideal_gas(0);
    set_fields({FIELD_DENSITY0, FIELD_ENERGY0, FIELD_PRESSURE, FIELD_VISCOSITY, FIELD_DENSITY1, FIELD_ENERGY1,
                FIELD_XVEL0, FIELD_YVEL0, FIELD_XVEL1, FIELD_YVEL1});
    update_halo(fields, 2);
    field_summary();
  }

  // One hydro cycle (clover_leaf.cpp:185-212). Returns true when complete.
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

}  // namespace clover
}  // namespace opsb

extern "C" int ops_b200_app_cloverleaf(const ops_b200_clover_deck *deck, int warmup_steps, double *summaries,
                                       int max_summaries, int *n_summaries, double *device_seconds,
                                       const char *dump_dir) {
  using namespace opsb;
  return capi_guard([&] {
    if (!deck || warmup_steps < 0) throw Error(E_ARG, "bad CloverLeaf arguments");
    if (deck->x_cells < 2 || deck->y_cells < 2) throw Error(E_ARG, "x_cells and y_cells must be >= 2");
    Runtime &r = Runtime::get();
    if (!r.initialized()) r.init(0, 0);
    ReleaseScope scope(r);
    const Runtime::Mark &mk = scope.mark();
    clover::Clover c(r);
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
