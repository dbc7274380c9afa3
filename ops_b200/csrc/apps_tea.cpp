// TeaLeaf 2D driver on the OPS-B200 runtime: the loop sequence of the
// reference app (apps/c/TeaLeaf/diffuse.cpp:78-148, start.cpp:46-110,
// tea_solve.cpp:37-418 and the files they call, cited per function) for the
// Jacobi, CG, Chebyshev and PPCG solvers (no preconditioner or the Jacobi
// diagonal one), with the deck passed as a struct instead of tea.in.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/ops_b200.h"
#include "clover_common.h"
#include "heat_pcg.h"
#include "runtime.h"

namespace opsb {
int capi_guard(const std::function<int()> &f);

namespace tea {

enum { FIELD_DENSITY = 0, FIELD_ENERGY0, FIELD_ENERGY1, FIELD_U, FIELD_P, FIELD_SD, FIELD_R, FIELD_Z, NUM_FIELDS };
enum { CONDUCTIVITY = 1, RECIP_CONDUCTIVITY = 2 };
enum { TL_PREC_NONE = 1, TL_PREC_JAC_DIAG = 2 };

struct Tea {
  Runtime &r;
  double g_small = 1.0e-16, g_big = 1.0e+21;
  double dt = 0, dtinit = 0.1, currtime = 0, end_time = 10.0, eps = 1e-10;
  int end_step = 640000, summary_frequency = 10, max_iters = 1000, coefficient = CONDUCTIVITY;
  int prec = TL_PREC_NONE, use_cg = 0, reflective_boundary = 0, check_result = 0;
  // Chebyshev / PPCG (read_input.cpp:93-101, tea_solve.cpp:37-38): the
  // eigenvalue estimate is made once per run (`first`) and reused by every
  // later solve; theta persists with it.
  int use_cheby = 0, use_ppcg = 0, ch_cg_presteps = 25, ppcg_inner_steps = -1, ppcg_active = 0, first = 1;
  double ch_cg_epslim = 1.0, eigmin = 0.0, eigmax = 0.0, theta = 0.0, cn = 0.0;
  int step = 0, complete = 0;
  int g_rect = clover::G_RECT, g_circ = clover::G_CIRC, g_point = clover::G_POINT;
  int number_of_states = 0;
  clover::state_type states[clover::kMaxStates];
  clover::grid_type grid;
  clover::field_type field;
  int fields[NUM_FIELDS] = {0};

  int tea_grid = -1;
  int density, energy0, energy1, u, u0, vector_r, vector_rstore, vector_rtemp, vector_Mi, vector_w, vector_z;
  int vector_utemp, vector_Kx, vector_Ky, vector_p, vector_sd, tri_cp, tri_bfp;
  int volume, xarea, yarea, cellx, celldx, celly, celldy, vertexx, vertexdx, vertexy, vertexdy, xx, yy;
  int S2D_00, S2D_00_P10, S2D_00_0P1, S2D_00_M10, S2D_00_0M1, S2D_00_0M1_M10_P10_0P1, S2D_00_M10_0M1;
  int S2D_00_P30, S2D_00_0P3, S2D_00_M30, S2D_00_0M3;
  int S2D_00_STRID2D_X, S2D_00_STRID2D_Y, S2D_00_P10_STRID2D_X, S2D_00_0P1_STRID2D_Y;
  int S2D_00_P10_M10_STRID2D_X, S2D_00_0P1_0M1_STRID2D_Y;
  int red_vol, red_mass, red_ie, red_temp;

  std::vector<double> summaries;  // step, time, vol, mass, ie, temp
  std::vector<double> solves;     // per solve: OPS_B200_TEA_SOLVE_COLS values
  int fused = 0, mixed = 0, true_stop = 0;
  double delta = 0.1;
  heat::Solver solver;
  cudaEvent_t ev_solve[2] = {nullptr, nullptr};

  explicit Tea(Runtime &rt) : r(rt) {
    memset(states, 0, sizeof(states));
    memset(&grid, 0, sizeof(grid));
    memset(&field, 0, sizeof(field));
    for (cudaEvent_t &e : ev_solve) OPSB_CUDA(cudaEventCreate(&e));
  }
  ~Tea() {
    for (cudaEvent_t e : ev_solve)
      if (e) cudaEventDestroy(e);
  }

  PrefixedLoops loops{"tealeaf/"};
  void loop(const char *k, const int *range, std::initializer_list<Arg> a) {
    r.par_loop(loops.get(k), k, tea_grid, 2, range, a.begin(), (int)a.size());
  }
  Arg dat(int d, int s, int acc) { return arg_dat(d, 1, s, acc); }
  int stencil(int points, std::initializer_list<int> offs, const char *name) {
    std::vector<int> o(offs);
    return r.decl_stencil(2, points, o.data(), nullptr, name);
  }
  int strided(int points, std::initializer_list<int> offs, std::initializer_list<int> stride, const char *name) {
    std::vector<int> o(offs), s(stride);
    return r.decl_stencil(2, points, o.data(), s.data(), name);
  }
  void set_fields(std::initializer_list<int> on) {
    for (int i = 0; i < NUM_FIELDS; i++) fields[i] = 0;
    for (int i : on) fields[i] = 1;
  }

  // read_input.cpp:70-378 (values already parsed)
  void read_input(const ops_b200_tea_deck &d) {
    grid.xmin = d.xmin; grid.ymin = d.ymin; grid.xmax = d.xmax; grid.ymax = d.ymax;
    grid.x_cells = d.x_cells; grid.y_cells = d.y_cells;
    dtinit = d.initial_timestep; end_time = d.end_time; end_step = d.end_step;
    summary_frequency = d.summary_frequency; max_iters = d.max_iters; eps = d.eps;
    coefficient = d.coefficient == 2 ? RECIP_CONDUCTIVITY : CONDUCTIVITY;
    prec = d.preconditioner == 1 ? TL_PREC_JAC_DIAG : TL_PREC_NONE;
    use_cg = d.solver == 1;
    use_cheby = d.solver == 2;
    use_ppcg = d.solver == 3;
    ch_cg_presteps = d.ch_cg_presteps;
    ch_cg_epslim = d.ch_cg_epslim;
    ppcg_inner_steps = d.ppcg_inner_steps;
    if (ppcg_inner_steps == -1)  // read_input.cpp:351-354
      ppcg_inner_steps = 4 * (int)(sqrt(sqrt((double)(d.x_cells * d.y_cells))));
    reflective_boundary = d.reflective_boundary;
    check_result = d.check_result;
    number_of_states = d.number_of_states;
    if (number_of_states < 1 || number_of_states > 24) throw Error(E_ARG, "1..24 states are supported");
    if (d.solver < 0 || d.solver > 3)
      throw Error(E_UNSUPPORTED, "solver must be 0 (Jacobi), 1 (CG), 2 (Chebyshev) or 3 (PPCG)");
    if (d.fused && d.solver != 1) throw Error(E_ARG, "fused solves need solver = 1 (CG)");
    fused = d.fused != 0;
    mixed = d.mixed != 0;
    true_stop = d.true_residual_stop != 0;
    delta = d.reliable_delta;
    if ((mixed || true_stop) && !fused) throw Error(E_ARG, "mixed and true_residual_stop need fused = 1");
    if (fused && reflective_boundary) throw Error(E_UNSUPPORTED, "fused solves need reflective_boundary = 0");
    if (mixed && !(delta > 0.0 && delta < 1.0)) throw Error(E_ARG, "reliable_delta must be in (0, 1)");
    for (int i = 0; i < number_of_states; i++) {
      const ops_b200_clover_state &s = d.states[i];
      states[i].defined = 1;
      states[i].density = s.density; states[i].energy = s.energy;
      states[i].geometry = s.geometry;
      states[i].xmin = s.xmin; states[i].xmax = s.xmax; states[i].ymin = s.ymin; states[i].ymax = s.ymax;
      states[i].radius = s.radius;
    }
    field.x_min = 1; field.y_min = 1;
    field.x_max = grid.x_cells + 1; field.y_max = grid.y_cells + 1;
    field.left = 0; field.bottom = 0;
    float dx = (grid.xmax - grid.xmin) / (float)(grid.x_cells);
    float dy = (grid.ymax - grid.ymin) / (float)(grid.y_cells);
    for (int i = 0; i < number_of_states; i++) {
      states[i].xmin = states[i].xmin + (dx / 100.00);
      states[i].ymin = states[i].ymin + (dy / 100.00);
      states[i].xmax = states[i].xmax - (dx / 100.00);
      states[i].ymax = states[i].ymax - (dy / 100.00);
    }
  }

  // build_field.cpp:37-178
  void build_field() {
    const int x_cells = grid.x_cells, y_cells = grid.y_cells;
    tea_grid = r.decl_block(2, "clover grid");
    int d_p[2] = {1, 1}, d_m[2] = {-1, -1}, size[2] = {x_cells, y_cells}, base[2] = {1, 1};
    auto D = [&](const char *n) { return r.decl_dat(tea_grid, 1, size, base, d_m, d_p, nullptr, 8, "double", n); };
    density = D("density"); energy0 = D("energy0"); energy1 = D("energy1"); u = D("u"); u0 = D("u0");
    vector_r = D("vector_r"); vector_rstore = D("vector_rstore"); vector_rtemp = D("vector_rtemp");
    vector_Mi = D("vector_Mi"); vector_w = D("vector_w"); vector_z = D("vector_z"); vector_utemp = D("vector_utemp");
    vector_Kx = D("vector_Kx"); vector_Ky = D("vector_Ky"); vector_p = D("vector_p"); vector_sd = D("vector_sd");
    tri_cp = D("tri_cp"); tri_bfp = D("tri_bfp");
    base[0] = -1; base[1] = -1;
    size[0] = x_cells + 4; size[1] = y_cells + 4;
    volume = D("volume");
    size[0] = x_cells + 5; size[1] = y_cells + 4;
    xarea = D("xarea");
    size[0] = x_cells + 4; size[1] = y_cells + 5;
    yarea = D("yarea");
    auto E = [&](int sx, int sy, int mx, int my, int px, int py, int bx, int by, const char *type, const char *n) {
      int sz[2] = {sx, sy}, dm[2] = {mx, my}, dp[2] = {px, py}, b[2] = {bx, by};
      return r.decl_dat(tea_grid, 1, sz, b, dm, dp, nullptr, 0, type, n);
    };
    cellx = E(x_cells + 4, 1, -2, 0, 2, 0, -1, 0, "double", "cellx");
    celldx = E(x_cells + 4, 1, -2, 0, 2, 0, -1, 0, "double", "celldx");
    celly = E(1, y_cells + 4, 0, -2, 0, 2, 0, -1, "double", "celly");
    celldy = E(1, y_cells + 4, 0, -2, 0, 2, 0, -1, "double", "celldy");
    vertexx = E(x_cells + 5, 1, -2, 0, 2, 0, -1, 0, "double", "vertexx");
    vertexdx = E(x_cells + 5, 1, -2, 0, 2, 0, -1, 0, "double", "vertexdx");
    vertexy = E(1, y_cells + 5, 0, -2, 0, 2, 0, -1, "double", "vertexy");
    vertexdy = E(1, y_cells + 5, 0, -2, 0, 2, 0, -1, "double", "vertexdy");
    xx = E(x_cells + 5, 1, -2, 0, 2, 0, 0, 0, "int", "xx");
    yy = E(1, y_cells + 5, 0, -2, 0, 2, 0, 0, "int", "yy");

    S2D_00 = stencil(1, {0, 0}, "00");
    S2D_00_P10 = stencil(2, {0, 0, 1, 0}, "0,0:1,0");
    S2D_00_0P1 = stencil(2, {0, 0, 0, 1}, "0,0:0,1");
    S2D_00_M10 = stencil(2, {0, 0, -1, 0}, "0,0:-1,0");
    S2D_00_0M1 = stencil(2, {0, 0, 0, -1}, "0,0:0,-1");
    S2D_00_0M1_M10_P10_0P1 = stencil(5, {0, 0, 0, -1, -1, 0, 1, 0, 0, 1}, "5pt");
    S2D_00_M10_0M1 = stencil(3, {0, 0, -1, 0, 0, -1}, "0,0:-1,0:0,-1");
    S2D_00_P30 = stencil(2, {0, 0, 3, 0}, "0,0:3,0");
    S2D_00_0P3 = stencil(2, {0, 0, 0, 3}, "0,0:0,3");
    S2D_00_M30 = stencil(2, {0, 0, -3, 0}, "0,0:-3,0");
    S2D_00_0M3 = stencil(2, {0, 0, 0, -3}, "0,0:0,-3");
    S2D_00_STRID2D_X = strided(1, {0, 0}, {1, 0}, "s2D_00_stride2D_x");
    S2D_00_STRID2D_Y = strided(1, {0, 0}, {0, 1}, "s2D_00_stride2D_y");
    S2D_00_P10_STRID2D_X = strided(2, {0, 0, 1, 0}, {1, 0}, "s2D_00_P10_stride2D_x");
    S2D_00_0P1_STRID2D_Y = strided(2, {0, 0, 0, 1}, {0, 1}, "s2D_00_0P1_stride2D_y");
    S2D_00_P10_M10_STRID2D_X = strided(3, {0, 0, 1, 0, -1, 0}, {1, 0}, "self_stride2D_x");
    S2D_00_0P1_0M1_STRID2D_Y = strided(3, {0, 0, 0, 1, 0, -1}, {0, 1}, "self_stride2D_y");
    red_vol = r.decl_reduction(8, "double", "vol");
    red_mass = r.decl_reduction(8, "double", "mass");
    red_ie = r.decl_reduction(8, "double", "ie");
    red_temp = r.decl_reduction(8, "double", "temp");
  }

  // initialise_chunk.cpp:40-176
  void initialise_chunk() {
    const int x_min = field.x_min, x_max = field.x_max, y_min = field.y_min, y_max = field.y_max;
    const int x_cells = grid.x_cells, y_cells = grid.y_cells;
    int range[] = {x_min, x_max, y_min, y_max};
    for (int d : {density, energy0, energy1, u, u0, vector_r, vector_rstore, vector_rtemp, vector_Mi, vector_w,
                  vector_z, vector_utemp, vector_Kx, vector_Ky, vector_p, vector_sd, tri_cp, tri_bfp})
      loop("initialise_chunk_kernel_zero", range, {dat(d, S2D_00, ACC_WRITE)});
    int rf1[] = {-2, x_cells + 2, -2, y_cells + 2};
    loop("initialise_chunk_kernel_zero", rf1, {dat(volume, S2D_00, ACC_WRITE)});
    int rf2[] = {-2, x_cells + 3, -2, y_cells + 2};
    loop("initialise_chunk_kernel_zero", rf2, {dat(xarea, S2D_00, ACC_WRITE)});
    int rf3[] = {-2, x_cells + 2, -2, y_cells + 3};
    loop("initialise_chunk_kernel_zero", rf3, {dat(yarea, S2D_00, ACC_WRITE)});
    int rangex[] = {x_min - 2, x_max + 2, y_min - 2, y_max + 2};
    loop("initialise_chunk_kernel_zero_x", rangex, {dat(cellx, S2D_00_STRID2D_X, ACC_WRITE)});
    loop("initialise_chunk_kernel_zero_x", rangex, {dat(celldx, S2D_00_STRID2D_X, ACC_WRITE)});
    rangex[1]++;
    loop("initialise_chunk_kernel_zero_x", rangex, {dat(vertexx, S2D_00_STRID2D_X, ACC_WRITE)});
    loop("initialise_chunk_kernel_zero_x", rangex, {dat(vertexdx, S2D_00_STRID2D_X, ACC_WRITE)});
    int rangey2[] = {x_min - 2, x_max + 2, y_min - 2, y_max + 2};
    loop("initialise_chunk_kernel_zero_y", rangey2, {dat(celly, S2D_00_STRID2D_Y, ACC_WRITE)});
    loop("initialise_chunk_kernel_zero_y", rangey2, {dat(celldy, S2D_00_STRID2D_Y, ACC_WRITE)});
    rangey2[3]++;
    loop("initialise_chunk_kernel_zero_y", rangey2, {dat(vertexy, S2D_00_STRID2D_Y, ACC_WRITE)});
    loop("initialise_chunk_kernel_zero_y", rangey2, {dat(vertexdy, S2D_00_STRID2D_Y, ACC_WRITE)});
    int rangefull[] = {x_min - 2, x_max + 3, y_min - 2, y_max + 3};
    loop("initialise_chunk_kernel_xx", rangefull, {dat(xx, S2D_00_STRID2D_X, ACC_WRITE), arg_idx()});
    loop("initialise_chunk_kernel_yy", rangefull, {dat(yy, S2D_00_STRID2D_Y, ACC_WRITE), arg_idx()});
    loop("initialise_chunk_kernel_x", rangex,
         {dat(vertexx, S2D_00_STRID2D_X, ACC_WRITE), dat(xx, S2D_00_STRID2D_X, ACC_READ),
          dat(vertexdx, S2D_00_STRID2D_X, ACC_WRITE)});
    loop("initialise_chunk_kernel_y", rangey2,
         {dat(vertexy, S2D_00_STRID2D_Y, ACC_WRITE), dat(yy, S2D_00_STRID2D_Y, ACC_READ),
          dat(vertexdy, S2D_00_STRID2D_Y, ACC_WRITE)});
    rangex[0] = x_min - 2; rangex[1] = x_max + 2; rangex[2] = y_min - 2; rangex[3] = y_max + 2;
    loop("initialise_chunk_kernel_cellx", rangex,
         {dat(vertexx, S2D_00_P10_STRID2D_X, ACC_READ), dat(cellx, S2D_00_STRID2D_X, ACC_WRITE),
          dat(celldx, S2D_00_STRID2D_X, ACC_WRITE)});
    int rangey[] = {x_min - 2, x_max + 3, y_min - 2, y_max + 2};
    loop("initialise_chunk_kernel_celly", rangey,
         {dat(vertexy, S2D_00_0P1_STRID2D_Y, ACC_READ), dat(celly, S2D_00_STRID2D_Y, ACC_WRITE),
          dat(celldy, S2D_00_STRID2D_Y, ACC_WRITE)});
    int rangexy[] = {x_min - 2, x_max + 2, y_min - 2, y_max + 2};
    loop("initialise_chunk_kernel_volume", rangexy,
         {dat(volume, S2D_00, ACC_WRITE), dat(celldy, S2D_00_STRID2D_Y, ACC_READ), dat(xarea, S2D_00, ACC_WRITE),
          dat(celldx, S2D_00_STRID2D_X, ACC_READ), dat(yarea, S2D_00, ACC_WRITE)});
  }

  void generate() {  // generate.cpp:36-58
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("generate_chunk_kernel", rng,
         {dat(vertexx, S2D_00_P10_M10_STRID2D_X, ACC_READ), dat(vertexy, S2D_00_0P1_0M1_STRID2D_Y, ACC_READ),
          dat(energy0, S2D_00, ACC_WRITE), dat(density, S2D_00, ACC_WRITE), dat(u, S2D_00, ACC_WRITE),
          dat(cellx, S2D_00_P10_M10_STRID2D_X, ACC_READ), dat(celly, S2D_00_0P1_0M1_STRID2D_Y, ACC_READ)});
  }

  // update_halo.cpp:36-149: only with reflective boundaries.
  void update_halo(const int *f, int depth) {
    if (reflective_boundary != 1) return;
    if (!(f[FIELD_DENSITY] || f[FIELD_ENERGY0] || f[FIELD_ENERGY1] || f[FIELD_U] || f[FIELD_P] || f[FIELD_SD])) return;
    const int x_min = field.x_min, x_max = field.x_max, y_min = field.y_min, y_max = field.y_max;
    Arg gbl = arg_gbl(f, NUM_FIELDS, 4, ACC_READ);
    auto k1 = [&](const char *k, const int *rng, int st) {
      loop(k, rng,
           {arg_dat_opt(density, 1, st, ACC_RW, f[FIELD_DENSITY]), arg_dat_opt(energy0, 1, st, ACC_RW, f[FIELD_ENERGY0]),
            arg_dat_opt(energy1, 1, st, ACC_RW, f[FIELD_ENERGY1]), arg_dat_opt(u, 1, st, ACC_RW, f[FIELD_U]),
            arg_dat_opt(vector_p, 1, st, ACC_RW, f[FIELD_P]), arg_dat_opt(vector_sd, 1, st, ACC_RW, f[FIELD_SD]),
            gbl});
    };
    int b2[] = {x_min - depth, x_max + depth, y_min - 2, y_min - 1};
    if (depth == 2) k1("update_halo_kernel1_b2", b2, S2D_00_0P3);
    int b1[] = {x_min - depth, x_max + depth, y_min - 1, y_min};
    k1("update_halo_kernel1_b1", b1, S2D_00_0P1);
    int t2[] = {x_min - depth, x_max + depth, y_max + 1, y_max + 2};
    if (depth == 2) k1("update_halo_kernel1_t2", t2, S2D_00_0M3);
    int t1[] = {x_min - depth, x_max + depth, y_max, y_max + 1};
    k1("update_halo_kernel1_t1", t1, S2D_00_0M1);
    int l2[] = {x_min - 2, x_min - 1, y_min - depth, y_max + depth};
    if (depth == 2) k1("update_halo_kernel1_l2", l2, S2D_00_P30);
    int l1[] = {x_min - 1, x_min, y_min - depth, y_max + depth};
    k1("update_halo_kernel1_l1", l1, S2D_00_P10);
    int r2[] = {x_max + 1, x_max + 2, y_min - depth, y_max + depth};
    if (depth == 2) k1("update_halo_kernel1_r2", r2, S2D_00_M30);
    int r1[] = {x_max, x_max + 1, y_min - depth, y_max + depth};
    k1("update_halo_kernel1_r1", r1, S2D_00_M10);
  }

  void set_field() {  // set_field.cpp:37-52
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("set_field_kernel", rng, {dat(energy0, S2D_00, ACC_READ), dat(energy1, S2D_00, ACC_WRITE)});
  }

  void field_summary() {  // field_summary.cpp:41-111
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("field_summary_kernel", rng,
         {dat(volume, S2D_00, ACC_READ), dat(density, S2D_00, ACC_READ), dat(energy1, S2D_00, ACC_READ),
          dat(u, S2D_00, ACC_READ), arg_reduce(red_vol, 1, ACC_INC), arg_reduce(red_mass, 1, ACC_INC),
          arg_reduce(red_ie, 1, ACC_INC), arg_reduce(red_temp, 1, ACC_INC)});
    double vol = 0, mass = 0, ie = 0, temp = 0;
    r.reduction_result(red_vol, &vol);
    r.reduction_result(red_mass, &mass);
    r.reduction_result(red_ie, &ie);
    r.reduction_result(red_temp, &temp);
    double row[6] = {(double)step, currtime, vol, mass, ie, temp};
    summaries.insert(summaries.end(), row, row + 6);
  }

  // tea_leaf_common.cpp:40-141
  void common_init(int halo_depth, double *rx, double *ry) {
    double dx = (grid.xmax - grid.xmin) / (double)grid.x_cells;
    double dy = (grid.xmax - grid.xmin) / (double)grid.x_cells;
    *rx = dt / (dx * dx);
    *ry = dt / (dy * dy);
    const int x_min = field.x_min, x_max = field.x_max, y_min = field.y_min, y_max = field.y_max;
    int rangexy[] = {x_min, x_max, y_min, y_max};
    int ext[] = {x_min - halo_depth + 1, x_max + halo_depth, y_min - halo_depth + 1, y_max + halo_depth};
    int ext2[] = {x_min - halo_depth, x_max + halo_depth, y_min - halo_depth, y_max + halo_depth};
    loop("tea_leaf_common_init_u_u0_kernel", rangexy,
         {dat(u, S2D_00, ACC_WRITE), dat(u0, S2D_00, ACC_WRITE), dat(energy1, S2D_00, ACC_READ),
          dat(density, S2D_00, ACC_READ)});
    if (coefficient == RECIP_CONDUCTIVITY)
      loop("tea_leaf_recip_kernel", ext2, {dat(vector_w, S2D_00, ACC_WRITE), dat(density, S2D_00, ACC_READ)});
    else
      loop("tea_leaf_yeqx_kernel", ext2, {dat(vector_w, S2D_00, ACC_WRITE), dat(density, S2D_00, ACC_READ)});
    loop("tea_leaf_common_init_Kx_Ky_kernel", ext,
         {dat(vector_Kx, S2D_00, ACC_WRITE), dat(vector_Ky, S2D_00, ACC_WRITE), dat(vector_w, S2D_00_M10_0M1, ACC_READ)});
    if (reflective_boundary == 0) {
      int left[] = {x_min - halo_depth, x_min + 1, y_min - halo_depth, y_max + halo_depth};
      loop("tea_leaf_init_zero_kernel", left, {dat(vector_Kx, S2D_00, ACC_WRITE)});
      int right[] = {x_max, x_max + halo_depth, y_min - halo_depth, y_max + halo_depth};
      loop("tea_leaf_init_zero_kernel", right, {dat(vector_Kx, S2D_00, ACC_WRITE)});
      int bottom[] = {x_min - halo_depth, x_max + halo_depth, y_min - halo_depth, y_min + 1};
      loop("tea_leaf_init_zero_kernel", bottom, {dat(vector_Ky, S2D_00, ACC_WRITE)});
      int top[] = {x_min - halo_depth, x_max + halo_depth, y_max, y_max + halo_depth};
      loop("tea_leaf_init_zero_kernel", top, {dat(vector_Ky, S2D_00, ACC_WRITE)});
    }
    if (prec == TL_PREC_JAC_DIAG) {  // tea_diag_init, tea_leaf_common.cpp:243-258
      int e1[] = {x_min - halo_depth + 1, x_max + halo_depth - 1, y_min - halo_depth + 1, y_max + halo_depth - 1};
      loop("tea_leaf_common_init_diag_init_kernel", e1,
           {dat(vector_Mi, S2D_00, ACC_WRITE), dat(vector_Kx, S2D_00_P10, ACC_READ),
            dat(vector_Ky, S2D_00_0P1, ACC_READ), arg_gbl(rx, 1, 8, ACC_READ), arg_gbl(ry, 1, 8, ACC_READ)});
    }
    loop("tea_leaf_common_init_kernel", rangexy,
         {dat(vector_w, S2D_00, ACC_WRITE), dat(vector_r, S2D_00, ACC_WRITE), dat(vector_Kx, S2D_00_P10, ACC_READ),
          dat(vector_Ky, S2D_00_0P1, ACC_READ), dat(u, S2D_00_0M1_M10_P10_0P1, ACC_READ), arg_gbl(rx, 1, 8, ACC_READ),
          arg_gbl(ry, 1, 8, ACC_READ)});
  }

  void calc_residual(double rx, double ry) {  // tea_leaf_common.cpp:160-182
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("tea_leaf_common_residual_kernel", rng,
         {dat(vector_r, S2D_00, ACC_WRITE), dat(vector_Kx, S2D_00_P10, ACC_READ), dat(vector_Ky, S2D_00_0P1, ACC_READ),
          dat(u, S2D_00_0M1_M10_P10_0P1, ACC_READ), dat(u0, S2D_00, ACC_READ), arg_gbl(&rx, 1, 8, ACC_READ),
          arg_gbl(&ry, 1, 8, ACC_READ)});
  }

  double calc_2norm(int arr) {  // tea_leaf_common.cpp:184-211
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("tea_leaf_norm2_kernel", rng, {dat(arr, S2D_00, ACC_READ), arg_reduce(red_temp, 1, ACC_INC)});
    double norm = 0.0;
    r.reduction_result(red_temp, &norm);
    return norm;
  }

  void diag_solve() {  // tea_leaf_common.cpp:260-280 (z = Mi r over the range extended by the halo)
    int rng[] = {field.x_min - 1, field.x_max + 1, field.y_min - 1, field.y_max + 1};
    loop("tea_leaf_zeqxty_kernel", rng,
         {dat(vector_z, S2D_00, ACC_WRITE), dat(vector_Mi, S2D_00, ACC_READ), dat(vector_r, S2D_00, ACC_READ)});
  }

  double cg_init() {  // tea_leaf_cg.cpp:53-101
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("tea_leaf_init_zero2_kernel", rng, {dat(vector_p, S2D_00, ACC_WRITE), dat(vector_z, S2D_00, ACC_WRITE)});
    if (prec != TL_PREC_NONE) {
      diag_solve();
      loop("tea_leaf_yeqx_kernel", rng, {dat(vector_p, S2D_00, ACC_WRITE), dat(vector_z, S2D_00, ACC_READ)});
    } else {
      loop("tea_leaf_yeqx_kernel", rng, {dat(vector_p, S2D_00, ACC_WRITE), dat(vector_r, S2D_00, ACC_READ)});
    }
    loop("tea_leaf_dot_kernel", rng,
         {dat(vector_r, S2D_00, ACC_READ), dat(vector_p, S2D_00, ACC_READ), arg_reduce(red_temp, 1, ACC_INC)});
    double rro = 0.0;
    r.reduction_result(red_temp, &rro);
    return rro;
  }

  double cg_calc_w(double rx, double ry) {  // tea_leaf_cg.cpp:103-127
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("tea_leaf_cg_calc_w_reduce_kernel", rng,
         {dat(vector_w, S2D_00, ACC_WRITE), dat(vector_Kx, S2D_00_P10, ACC_READ), dat(vector_Ky, S2D_00_0P1, ACC_READ),
          dat(vector_p, S2D_00_0M1_M10_P10_0P1, ACC_READ), arg_gbl(&rx, 1, 8, ACC_READ), arg_gbl(&ry, 1, 8, ACC_READ),
          arg_reduce(red_temp, 1, ACC_INC)});
    double pw = 0.0;
    r.reduction_result(red_temp, &pw);
    return pw;
  }

  double cg_calc_ur(double alpha) {  // tea_leaf_cg.cpp:129-186
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    if (prec != TL_PREC_NONE) {
      loop("tea_leaf_axpy_kernel", rng,
           {dat(u, S2D_00, ACC_INC), dat(vector_p, S2D_00, ACC_READ), arg_gbl(&alpha, 1, 8, ACC_READ)});
      double malpha = -1.0 * alpha;
      loop("tea_leaf_axpy_kernel", rng,
           {dat(vector_r, S2D_00, ACC_INC), dat(vector_w, S2D_00, ACC_READ), arg_gbl(&malpha, 1, 8, ACC_READ)});
      diag_solve();
      loop("tea_leaf_dot_kernel", rng,
           {dat(vector_r, S2D_00, ACC_READ), dat(vector_z, S2D_00, ACC_READ), arg_reduce(red_temp, 1, ACC_INC)});
    } else {
      loop("tea_leaf_axpy_kernel", rng,
           {dat(u, S2D_00, ACC_INC), dat(vector_p, S2D_00, ACC_READ), arg_gbl(&alpha, 1, 8, ACC_READ)});
      loop("tea_leaf_cg_calc_ur_r_reduce_kernel", rng,
           {dat(vector_r, S2D_00, ACC_INC), dat(vector_w, S2D_00, ACC_READ), arg_gbl(&alpha, 1, 8, ACC_READ),
            arg_reduce(red_temp, 1, ACC_INC)});
    }
    double rnn = 0.0;
    r.reduction_result(red_temp, &rnn);
    return rnn;
  }

  void cg_calc_p(double beta) {  // tea_leaf_cg.cpp:188-214
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    double one = 1.0;
    int src = (prec != TL_PREC_NONE || ppcg_active) ? vector_z : vector_r;
    loop("tea_leaf_axpby_kernel", rng,
         {dat(vector_p, S2D_00, ACC_RW), dat(src, S2D_00, ACC_READ), arg_gbl(&beta, 1, 8, ACC_READ),
          arg_gbl(&one, 1, 8, ACC_READ)});
  }

  double jacobi_solve(double rx, double ry) {  // tea_leaf_jacobi.cpp:40-70
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("tea_leaf_yeqx_kernel", rng, {dat(vector_r, S2D_00, ACC_WRITE), dat(u, S2D_00, ACC_READ)});
    loop("tea_leaf_jacobi_kernel", rng,
         {dat(u, S2D_00, ACC_WRITE), dat(vector_Kx, S2D_00_P10, ACC_READ), dat(vector_Ky, S2D_00_0P1, ACC_READ),
          dat(vector_r, S2D_00_0M1_M10_P10_0P1, ACC_READ), dat(u0, S2D_00, ACC_READ), arg_gbl(&rx, 1, 8, ACC_READ),
          arg_gbl(&ry, 1, 8, ACC_READ), arg_reduce(red_temp, 1, ACC_INC)});
    double error = 0.0;
    r.reduction_result(red_temp, &error);
    return error;
  }

  // ---- Chebyshev (tea_leaf_cheby.cpp) ------------------------------------
  // w = A u, r = u0 - w; p = (Mi r or r) / theta; u += p   (:43-96)
  void cheby_init(double rx, double ry) {
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    cheby_residual(rx, ry);
    int src = vector_r;
    if (prec != TL_PREC_NONE) {
      diag_solve();
      src = vector_z;
    }
    loop("tea_leaf_recip3_kernel", rng,
         {dat(vector_p, S2D_00, ACC_WRITE), dat(src, S2D_00, ACC_READ), arg_gbl(&theta, 1, 8, ACC_READ)});
    loop("tea_leaf_xpy_kernel", rng, {dat(u, S2D_00, ACC_INC), dat(vector_p, S2D_00, ACC_READ)});
  }
  void cheby_residual(double rx, double ry) {
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("tea_leaf_cheby_init_kernel", rng,
         {dat(vector_w, S2D_00, ACC_WRITE), dat(vector_r, S2D_00, ACC_WRITE), dat(vector_Kx, S2D_00_P10, ACC_READ),
          dat(vector_Ky, S2D_00_0P1, ACC_READ), dat(u, S2D_00_0M1_M10_P10_0P1, ACC_READ), dat(u0, S2D_00, ACC_READ),
          arg_gbl(&rx, 1, 8, ACC_READ), arg_gbl(&ry, 1, 8, ACC_READ)});
  }
  // r = u0 - A u; p = alpha_k p + beta_k (Mi r or r); u += p   (:98-151)
  void cheby_iterate(double rx, double ry, int k) {
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    cheby_residual(rx, ry);
    int src = vector_r;
    if (prec != TL_PREC_NONE) {
      diag_solve();
      src = vector_z;
    }
    loop("tea_leaf_axpby_kernel", rng,
         {dat(vector_p, S2D_00, ACC_RW), dat(src, S2D_00, ACC_READ), arg_gbl(&ch_alphas[k], 1, 8, ACC_READ),
          arg_gbl(&ch_betas[k], 1, 8, ACC_READ)});
    loop("tea_leaf_xpy_kernel", rng, {dat(u, S2D_00, ACC_INC), dat(vector_p, S2D_00, ACC_READ)});
  }

  // Eigenvalues of the symmetric tridiagonal matrix d[1..n] (diagonal),
  // e[2..n] (sub-diagonal) by the implicit QL method with Wilkinson shifts
  // (Numerical Recipes' tqli, the routine tea_leaf_cheby.cpp:153-211 calls),
  // overwriting d. The floating-point steps are those of the reference, so
  // the estimate rounds identically. Returns false when an eigenvalue needs
  // more than 30 sweeps.
  static bool ql_implicit(double *d, double *e, int n) {
    for (int i = 1; i < n; i++) e[i] = e[i + 1];
    e[n] = 0.0;
    for (int l = 1; l <= n; l++) {
      for (int sweep = 0;; sweep++) {
        int m = l;
        for (; m <= n - 1; m++) {  // first negligible off-diagonal at or after l
          double dd = fabs(d[m]) + fabs(d[m + 1]);
          if (fabs(e[m]) + dd == dd) break;
        }
        if (m == l) break;
        if (sweep == 30) return false;
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = sqrt(g * g + 1.0);
        g = d[m] - d[l] + e[l] / (g + (g < 0.0 ? -r : r));
        double s = 1.0, c = 1.0, p = 0.0;
        bool deflated = false;
        for (int i = m - 1; i >= l; i--) {  // chase the bulge with Givens rotations
          double f = s * e[i], b = c * e[i];
          r = sqrt(f * f + g * g);
          e[i + 1] = r;
          if (r == 0.0) {  // underflow: the matrix split, restart this eigenvalue
            d[i + 1] = d[i + 1] - p;
            e[m] = 0.0;
            deflated = true;
            break;
          }
          s = f / r;
          c = g / r;
          g = d[i + 1] - p;
          r = (d[i] - g) * s + 2.0 * c * b;
          p = s * r;
          d[i + 1] = g + p;
          g = c * r - b;
        }
        if (deflated) continue;
        d[l] = d[l] - p;
        e[l] = g;
        e[m] = 0.0;
      }
    }
    return true;
  }

  // Extreme eigenvalues of the Lanczos matrix that k CG steps define
  // (tea_leaf_cheby.cpp:213-254): T_jj = 1/alpha_j + beta_{j-1}/alpha_{j-1},
  // T_{j,j+1} = sqrt(beta_j)/alpha_j. The reference bubble-sorts the
  // eigenvalues (and would not terminate on two equal ones); a sort gives
  // the same extremes.
  void calc_eigenvalues(int k) {
    std::vector<double> d(max_iters + 2, 0.0), e(max_iters + 2, 0.0);
    for (int n = 1; n <= k; n++) {
      d[n] = 1.0 / cg_alphas[n];
      if (n > 1) d[n] = d[n] + cg_betas[n - 1] / cg_alphas[n - 1];
      if (n < k) e[n + 1] = sqrt(cg_betas[n]) / cg_alphas[n];
    }
    bool ok = ql_implicit(d.data(), e.data(), k);
    if (ok && k > 1) std::sort(d.begin() + 1, d.begin() + k + 1);
    eigmin = d[1];
    eigmax = d[k];
    if (!ok || eigmin < 0.0 || eigmax < 0.0) throw Error(E_STATE, "Error in calculating eigenvalues");
  }

  // Chebyshev recurrence coefficients for [eigmin, eigmax]   (:256-280)
  void calc_ch_coefs(int count) {
    theta = (eigmax + eigmin) / 2.0;
    double delta = (eigmax - eigmin) / 2.0;
    double sigma = theta / delta;
    double rho_old = 1.0 / sigma;
    for (int n = 1; n <= count; n++) {
      double rho_new = 1.0 / (2.0 * sigma - rho_old);
      ch_alphas[n] = rho_new * rho_old;
      ch_betas[n] = 2.0 * rho_new / delta;
      rho_old = rho_new;
    }
  }

  // First Chebyshev step and the iteration estimate   (:282-316)
  int cheby_first_step(double rx, double ry, double *error) {
    double bb = calc_2norm(u0);
    cheby_init(rx, ry);
    update_halo(fields, 1);
    cheby_iterate(rx, ry, 1);
    *error = calc_2norm(vector_r);
    double it_alpha = eps / 2.0 * sqrt(bb / (*error));
    double gamm = (sqrt(cn) - 1.0) / (sqrt(cn) + 1.0);
    return (int)round(log(it_alpha) / (log(gamm)));
  }

  // ---- PPCG (tea_leaf_ppcg.cpp) --------------------------------------------
  // Steps 2 and 3 of the re-initialisation when the polynomial takes over
  // (:85-152): step 2 refreshes z = Mi r, step 3 restarts p from z.
  double ppcg_init(int step) {
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    double rro = 0.0;
    if (step == 1)
      loop("tea_leaf_init_zero2_kernel", rng, {dat(vector_p, S2D_00, ACC_WRITE), dat(vector_z, S2D_00, ACC_WRITE)});
    else if (step == 3)
      loop("tea_leaf_init_zero_kernel", rng, {dat(vector_p, S2D_00, ACC_WRITE)});
    if (prec != TL_PREC_NONE || (ppcg_active && step == 3)) {
      if (step == 1 || step == 2) diag_solve();
      if (step == 1 || step == 3)
        loop("tea_leaf_yeqx_kernel", rng, {dat(vector_p, S2D_00, ACC_WRITE), dat(vector_z, S2D_00, ACC_READ)});
    } else if (step == 1) {
      loop("tea_leaf_yeqx_kernel", rng, {dat(vector_p, S2D_00, ACC_WRITE), dat(vector_r, S2D_00, ACC_READ)});
    }
    if (step == 1 || step == 3) {
      loop("tea_leaf_dot_kernel", rng,
           {dat(vector_p, S2D_00, ACC_READ), dat(vector_r, S2D_00, ACC_READ), arg_reduce(red_temp, 1, ACC_INC)});
      r.reduction_result(red_temp, &rro);
    }
    return rro;
  }

  // z <- the Chebyshev polynomial of degree ppcg_inner_steps applied to r
  // (:300-364, init_sd :51-83, inner :154-215). As in the reference, the
  // preconditioned variant refreshes z from r, not from rtemp, every step.
  void run_ppcg_inner_steps(double rx, double ry) {
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    int f[NUM_FIELDS] = {0};
    f[FIELD_U] = 1;
    update_halo(f, 1);
    double theta_r = 1.0 / theta;
    if (prec != TL_PREC_NONE)
      loop("tea_leaf_ppcg_init1_kernel", rng,
           {dat(vector_sd, S2D_00, ACC_WRITE), dat(vector_rtemp, S2D_00, ACC_WRITE),
            dat(vector_utemp, S2D_00, ACC_WRITE), dat(vector_z, S2D_00, ACC_READ), dat(vector_r, S2D_00, ACC_READ),
            arg_gbl(&theta_r, 1, 8, ACC_READ)});
    else
      loop("tea_leaf_ppcg_init2_kernel", rng,
           {dat(vector_sd, S2D_00, ACC_WRITE), dat(vector_rtemp, S2D_00, ACC_WRITE),
            dat(vector_utemp, S2D_00, ACC_WRITE), dat(vector_r, S2D_00, ACC_READ), arg_gbl(&theta_r, 1, 8, ACC_READ)});
    for (int k = 1; k <= ppcg_inner_steps; k++) {
      int g[NUM_FIELDS] = {0};
      g[FIELD_SD] = 1;
      g[FIELD_R] = 1;
      update_halo(g, 1);
      loop("tea_leaf_ppcg_inner1_kernel", rng,
           {dat(vector_rtemp, S2D_00, ACC_INC), dat(vector_Kx, S2D_00_P10, ACC_READ),
            dat(vector_Ky, S2D_00_0P1, ACC_READ), dat(vector_sd, S2D_00_0M1_M10_P10_0P1, ACC_READ),
            arg_gbl(&rx, 1, 8, ACC_READ), arg_gbl(&ry, 1, 8, ACC_READ)});
      int src = vector_rtemp;
      if (prec != TL_PREC_NONE) {
        diag_solve();
        src = vector_z;
      }
      loop("tea_leaf_ppcg_inner2_kernel", rng,
           {dat(vector_sd, S2D_00, ACC_RW), dat(vector_utemp, S2D_00, ACC_INC), dat(src, S2D_00, ACC_READ),
            arg_gbl(&ch_alphas[k], 1, 8, ACC_READ), arg_gbl(&ch_betas[k], 1, 8, ACC_READ)});
    }
    loop("tea_leaf_yeqx_kernel", rng, {dat(vector_z, S2D_00, ACC_WRITE), dat(vector_utemp, S2D_00, ACC_READ)});
  }

  double ppcg_calc_zrnorm() {  // :217-243
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    if (prec != TL_PREC_NONE || ppcg_active)
      loop("tea_leaf_dot_kernel", rng,
           {dat(vector_z, S2D_00, ACC_READ), dat(vector_r, S2D_00, ACC_READ), arg_reduce(red_temp, 1, ACC_INC)});
    else
      loop("tea_leaf_norm2_kernel", rng, {dat(vector_r, S2D_00, ACC_READ), arg_reduce(red_temp, 1, ACC_INC)});
    double norm = 0.0;
    r.reduction_result(red_temp, &norm);
    return norm;
  }

  double ppcg_calc_rrn() {  // (r - rstore) . z, :275-298
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("tea_leaf_ppcg_reduce_kernel", rng,
         {dat(vector_rstore, S2D_00, ACC_READ), dat(vector_r, S2D_00, ACC_READ), dat(vector_z, S2D_00, ACC_READ),
          arg_reduce(red_temp, 1, ACC_INC)});
    double rrn = 0.0;
    r.reduction_result(red_temp, &rrn);
    return rrn;
  }

  std::vector<double> cg_alphas, cg_betas, ch_alphas, ch_betas;

  double *interior(int d) {
    Dat &x = r.dat(d);
    return reinterpret_cast<double *>(x.origin_ptr()) + field.x_min + (long long)field.y_min * x.pitch;
  }

  // The CG solve as the device-resident iteration of heat_pcg.cu: the same
  // coefficient set-up loops, then the solver on the dats' storage.
  void tea_leaf_fused(double rx, double ry) {
    // the fused solver addresses the whole field on one GPU
    if (r.partitioned() && r.nranks() > 1)
      throw Error(E_UNSUPPORTED, "fused heat solves do not run on a block partitioned across ranks");
    r.execute();
    heat::Field2D f;
    f.nx = grid.x_cells;
    f.ny = grid.y_cells;
    f.pitch = r.dat(u).pitch;
    for (int d : {vector_Kx, vector_Ky, u0, u, vector_r, vector_w, vector_p, vector_z, vector_Mi})
      if (r.dat(d).pitch != f.pitch) throw Error(E_STATE, "fused heat solve: fields differ in pitch");
    f.Kx = interior(vector_Kx);
    f.Ky = interior(vector_Ky);
    f.u0 = interior(u0);
    f.u = interior(u);
    f.r = interior(vector_r);
    f.w = interior(vector_w);
    f.p = interior(vector_p);
    f.z = interior(vector_z);
    f.Mi = interior(vector_Mi);
    heat::SolveStats st;
    const bool pre = prec != TL_PREC_NONE;
    if (mixed)
      solver.pcg_mixed(f, rx, ry, pre, eps, delta, max_iters, r.stream(), &st);
    else
      solver.pcg_fp64(f, rx, ry, pre, true_stop, eps, max_iters, r.stream(), &st);
    r.count_kernels(solver.launches());
    const double ir = st.initial_residual;
    double srow[OPS_B200_TEA_SOLVE_COLS] = {(double)st.iterations, ir, st.error / ir, -1.0, st.true_residual / ir,
                                            (double)st.outer, 0.0, 0.0, -1.0, 0.0, 0.0, -1.0};
    solves.insert(solves.end(), srow, srow + OPS_B200_TEA_SOLVE_COLS);
  }

  // tea_solve.cpp:40-398: Jacobi, CG, and Chebyshev / PPCG after CG
  // presteps; the solve record gets the reference's printed quantities.
  void tea_leaf() {
    double rx, ry, rro = 0.0;
    ppcg_active = 0;
    int cheby_calc_steps = 0, ch_switch_check = 0, ppcg_inner_iters = 0, est_itc = -1, max_cheby_iters = 0;
    int switched_at = -1;
    set_fields({FIELD_ENERGY1, FIELD_DENSITY});
    update_halo(fields, 1);
    common_init(1, &rx, &ry);
    if (use_cg && fused) {
      tea_leaf_fused(rx, ry);
      finalise();
      return;
    }
    set_fields({FIELD_U});
    update_halo(fields, 1);
    calc_residual(rx, ry);
    double initial_residual = calc_2norm(vector_r);
    double old_error = initial_residual;  // the squared norm, as tea_solve.cpp:106-108 has it
    initial_residual = sqrt(fabs(initial_residual));
    const bool krylov = use_cg || use_cheby || use_ppcg;
    if (krylov) {
      rro = cg_init();
      set_fields({FIELD_U, FIELD_P});
      update_halo(fields, 1);
      set_fields({FIELD_P});
    } else {
      set_fields({FIELD_U});
    }
    cg_alphas.assign(max_iters + 1, 0.0);
    cg_betas.assign(max_iters + 1, 0.0);
    double error = 0.0;
    int n;
    for (n = 1; n <= max_iters; n++) {
      if (ch_switch_check == 0) {  // :146-160
        if (cheby_calc_steps > 0)
          ch_switch_check = 1;
        else if (first == 0 && use_ppcg && n > 1)
          ch_switch_check = 1;
        else if (fabs(old_error) <= ch_cg_epslim && n >= ch_cg_presteps)
          ch_switch_check = 1;
      }
      if ((use_cheby || use_ppcg) && ch_switch_check) {
        if (cheby_calc_steps == 0) {  // :165-238
          max_cheby_iters = max_iters - n + 2;
          if (first) {
            calc_eigenvalues(n - 1);
            first = 0;
            eigmin = eigmin * 0.95;
            eigmax = eigmax * 1.05;
          }
          // room for max_cheby_iters = max_iters + 1 (a switch at n = 1) and
          // for the inner steps that also run on the Chebyshev path
          size_t len = (size_t)std::max(max_iters + 2, ppcg_inner_steps + 1);
          ch_alphas.assign(len, 0.0);
          ch_betas.assign(len, 0.0);
          if (use_cheby) {
            calc_ch_coefs(max_cheby_iters);
            set_fields({FIELD_U});
          } else {
            calc_ch_coefs(ppcg_inner_steps);
            ppcg_active = 1;
          }
          cn = eigmax / eigmin;
          switched_at = n;
          rro = ppcg_init(2);
          run_ppcg_inner_steps(rx, ry);
          ppcg_inner_iters = ppcg_inner_iters + ppcg_inner_steps;
          rro = ppcg_init(3);
          set_fields({FIELD_U, FIELD_P});
          update_halo(fields, 1);
          set_fields({FIELD_P});
        }
        if (use_cheby) {  // :240-256
          if (cheby_calc_steps == 0) {
            est_itc = cheby_first_step(rx, ry, &old_error);
            cheby_calc_steps = 1;
          } else {
            cheby_iterate(rx, ry, cheby_calc_steps);
            // the residual is only measured every 10th step past est_itc;
            // in between `error` keeps its last value (and is re-rooted below)
            if (n >= est_itc && n % 10 == 0) error = calc_2norm(vector_r);
          }
        } else {  // PPCG as flexible CG (:261-300)
          double pw = cg_calc_w(rx, ry);
          loop_yeqx(vector_rstore, vector_r);
          rro = ppcg_calc_zrnorm();
          double alpha = rro / pw;
          cg_calc_ur(alpha);
          run_ppcg_inner_steps(rx, ry);
          ppcg_inner_iters = ppcg_inner_iters + ppcg_inner_steps;
          double rrn = ppcg_calc_rrn();
          double beta = rrn / rro;
          cg_calc_p(beta);
          error = rrn;
          rro = rrn;
        }
        cheby_calc_steps = cheby_calc_steps + 1;
      } else if (krylov) {  // :305-330
        fields[FIELD_P] = 1;
        double pw = cg_calc_w(rx, ry);
        double alpha = rro / pw;
        cg_alphas[n] = alpha;
        double rrn = cg_calc_ur(alpha);
        double beta = rrn / rro;
        cg_betas[n] = beta;
        cg_calc_p(beta);
        error = rrn;
        rro = rrn;
      } else {
        error = jacobi_solve(rx, ry);
      }
      update_halo(fields, 1);
      error = sqrt(fabs(error));
      if (fabs(error) < eps * initial_residual) break;
      old_error = error;
    }
    double exact = -1.0;
    if (check_result) {
      set_fields({FIELD_U});
      update_halo(fields, 1);
      calc_residual(rx, ry);
      exact = sqrt(calc_2norm(vector_r)) / initial_residual;
    }
    // the reference reports n - 1 (tea_solve.cpp:386), also when the loop ran out
    const bool poly = switched_at > 0;
    double srow[OPS_B200_TEA_SOLVE_COLS] = {(double)(n - 1), initial_residual, error / initial_residual, exact, -1.0,
                                            0.0, 0.0, (double)ppcg_inner_iters, (double)switched_at,
                                            poly ? eigmin : 0.0, poly ? eigmax : 0.0, (double)est_itc};
    solves.insert(solves.end(), srow, srow + OPS_B200_TEA_SOLVE_COLS);
    finalise();
  }

  void loop_yeqx(int y, int x) {  // tea_leaf_ppcg_store_r, tea_leaf_ppcg.cpp:258-273
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("tea_leaf_yeqx_kernel", rng, {dat(y, S2D_00, ACC_WRITE), dat(x, S2D_00, ACC_READ)});
  }

  void finalise() {  // tea_leaf_finalise (tea_solve.cpp:400-418)
    int rng[] = {field.x_min, field.x_max, field.y_min, field.y_max};
    loop("tea_leaf_recip2_kernel", rng,
         {dat(energy1, S2D_00, ACC_WRITE), dat(u, S2D_00, ACC_READ), dat(density, S2D_00, ACC_READ)});
    set_fields({FIELD_ENERGY1});
    update_halo(fields, 1);
  }

  void setup(const ops_b200_tea_deck &deck) {  // initialise.cpp + start.cpp:44-110
    read_input(deck);
    currtime = 0.0;
    step = 0;
    dt = dtinit;
    build_field();
    r.partition("2D_BLOCK_DECOMPSE");  // build_field.cpp:252
    r.decl_const("tealeaf/field", 1, "field_type", &field);
    r.decl_const("tealeaf/grid", 1, "grid_type", &grid);
    r.decl_const("tealeaf/number_of_states", 1, "int", &number_of_states);
    r.decl_const("tealeaf/states", number_of_states, "state_type", states);
    r.decl_const("tealeaf/g_circ", 1, "int", &g_circ);
    r.decl_const("tealeaf/g_point", 1, "int", &g_point);
    r.decl_const("tealeaf/g_rect", 1, "int", &g_rect);
    initialise_chunk();
    generate();
    set_fields({FIELD_DENSITY, FIELD_ENERGY0, FIELD_ENERGY1});
    update_halo(fields, 1);
    set_field();
    field_summary();
  }

  bool cycle() {  // diffuse.cpp:83-130
    step = step + 1;
    dt = dtinit;  // timestep.cpp:37-54
    r.execute();
    OPSB_CUDA(cudaEventRecord(ev_solve[0], r.stream()));
    tea_leaf();
    r.execute();
    OPSB_CUDA(cudaEventRecord(ev_solve[1], r.stream()));
    OPSB_CUDA(cudaEventSynchronize(ev_solve[1]));
    float ms = 0.f;
    OPSB_CUDA(cudaEventElapsedTime(&ms, ev_solve[0], ev_solve[1]));
    solves[solves.size() - OPS_B200_TEA_SOLVE_COLS + 6] = ms * 1e-3;
    currtime = currtime + dt;
    if (summary_frequency != 0)
      if ((step % summary_frequency) == 0) field_summary();
    if ((currtime + g_small) > end_time || (step >= end_step)) {
      complete = 1;
      field_summary();
      return true;
    }
    return false;
  }
};

}  // namespace tea
}  // namespace opsb

extern "C" int ops_b200_app_tealeaf(const ops_b200_tea_deck *deck, double *summaries, int max_summaries,
                                    int *n_summaries, double *solves, int max_solves, int *n_solves,
                                    double *device_seconds, const char *dump_dir) {
  using namespace opsb;
  return capi_guard([&] {
    if (!deck) throw Error(E_ARG, "deck required");
    if (deck->x_cells < 2 || deck->y_cells < 2) throw Error(E_ARG, "x_cells and y_cells must be >= 2");
    Runtime &r = Runtime::get();
    if (!r.initialized()) r.init(0, 0);
    ReleaseScope scope(r);
    const Runtime::Mark &mk = scope.mark();
    tea::Tea t(r);
    t.setup(*deck);
    EventPair ev;
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    r.execute();
    OPSB_CUDA(cudaEventRecord(e0, r.stream()));
    while (!t.cycle()) {
    }
    r.execute();
    OPSB_CUDA(cudaEventRecord(e1, r.stream()));
    OPSB_CUDA(cudaEventSynchronize(e1));
    if (device_seconds) *device_seconds = ev.ms() * 1e-3;
    int n = (int)(t.summaries.size() / 6), ns = (int)(t.solves.size() / OPS_B200_TEA_SOLVE_COLS);
    if (n_summaries) *n_summaries = n;
    if (n_solves) *n_solves = ns;
    if (summaries) memcpy(summaries, t.summaries.data(), sizeof(double) * 6 * std::min(n, max_summaries));
    if (solves)
      memcpy(solves, t.solves.data(), sizeof(double) * OPS_B200_TEA_SOLVE_COLS * std::min(ns, max_solves));
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
