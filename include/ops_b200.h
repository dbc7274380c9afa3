/*
 * OPS-B200: C-ABI of the B200-native OPS execution backend.
 *
 * Plain C types only (handles are ints, data are pointers + sizes). Every
 * entry point returns 0 (or a non-negative handle) on success and a negative
 * OPS_B200_ERR_* code on failure; ops_b200_last_error() then describes it.
 * Each declaration names the reference OPS interface it stands in for
 * (paths relative to the OPS source tree).
 *
 * Threading: one host thread drives one process-wide instance, as in the
 * reference (ops/c/src/core/ops_instance.cpp:37). Loops are queued lazily and
 * run on one CUDA stream; ops_b200_reduction_result, the data-access calls
 * and ops_b200_execute are the synchronisation points.
 */
#ifndef OPS_B200_H
#define OPS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define OPS_B200_OK 0
#define OPS_B200_ERR_ARG (-1)          /* invalid argument or handle        */
#define OPS_B200_ERR_CUDA (-2)         /* CUDA runtime error / no device    */
#define OPS_B200_ERR_STATE (-3)        /* call not valid in current state   */
#define OPS_B200_ERR_NOTFOUND (-4)     /* unknown loop kernel name          */
#define OPS_B200_ERR_TIMEOUT (-5)      /* a bounded device-side wait expired */
#define OPS_B200_ERR_UNSUPPORTED (-6)  /* outside what the backend supports */

/* Access modes and argument kinds keep the reference's values
 * (ops/c/include/ops_lib_core.h:84-93). */
#define OPS_B200_READ 0
#define OPS_B200_WRITE 1
#define OPS_B200_RW 2
#define OPS_B200_INC 3
#define OPS_B200_MIN 4
#define OPS_B200_MAX 5
#define OPS_B200_ARG_GBL 0
#define OPS_B200_ARG_DAT 1
#define OPS_B200_ARG_IDX 2
#define OPS_B200_ARG_REDUCE 3
/* Memory spaces (ops_memspace, ops/c/include/ops_lib_core.h). */
#define OPS_B200_HOST 1
#define OPS_B200_DEVICE 2

/* Description of the last failure on this thread (never NULL). */
const char *ops_b200_last_error(void);

/* ops_init (ops/c/src/core/ops_dummy_singlenode.cpp:979): selects the CUDA
 * device and creates the instance. Fails with OPS_B200_ERR_CUDA when no GPU
 * is present; there is no CPU execution path. */
int ops_b200_init(int device, int diags);
/* ops_exit (ops/c/src/core/ops_lib_core.cpp): frees all device storage. */
int ops_b200_exit(void);

/* ops_decl_block (ops/c/include/ops_lib_core.h:611). Returns a block handle. */
int ops_b200_decl_block(int dims, const char *name);

/* ops_decl_dat -> ops_decl_dat_char (ops/c/include/ops_lib_core.h:647,
 * ops/c/src/core/ops_device_singlenode_common.cpp:44). size/base/d_m/d_p have
 * `dims` entries; the allocated extent is size - d_m + d_p per dimension.
 * `data` (may be NULL) holds that full extent, x fastest, and is copied.
 * Returns a dat handle. */
int ops_b200_decl_dat(int block, int dim, const int *size, const int *base, const int *d_m, const int *d_p,
                      const void *data, int type_size, const char *type, const char *name);

/* ops_decl_stencil / ops_decl_strided_stencil
 * (ops/c/src/core/ops_lib_core.cpp:640,689). `stride` may be NULL. */
int ops_b200_decl_stencil(int dims, int points, const int *stencil, const char *name);
int ops_b200_decl_strided_stencil(int dims, int points, const int *stencil, const int *stride, const char *name);
/* ops_decl_restrict_stencil / ops_decl_prolong_stencil
 * (ops/c/src/core/ops_lib_core.cpp:740-833): at loop point x a restrict
 * stencil addresses the (fine) dat at x * stride + offset, a prolong stencil
 * the (coarse) dat at floor(x / stride) + offset, per dimension -- the
 * addressing the reference generates for them in its MPI backend
 * (ops_translator_legacy/c/ops_gen_mpi_lazy.py:283-315), which is the only
 * one that gives them a meaning. Only loop kernels built with `mgrid = true`
 * accept them (OPS_B200_ERR_UNSUPPORTED otherwise). */
int ops_b200_decl_restrict_stencil(int dims, int points, const int *stencil, const int *stride, const char *name);
int ops_b200_decl_prolong_stencil(int dims, int points, const int *stencil, const int *stride, const char *name);

/* ops_decl_reduction_handle (ops/c/src/core/ops_lib_core.cpp:1119). */
int ops_b200_decl_reduction_handle(int size, const char *type, const char *name);

/* ops_decl_halo (ops/c/include/ops_lib_core.h:888, ops_lib_core.cpp:998):
 * a box of iter_size (block dims entries) copied from dat `from` to dat
 * `to`; dat dimension i walks box dimension |dir[i]| - 1, backwards when
 * dir[i] < 0, from logical index *_base[i]. The dats may live on different
 * blocks and differ in type only as float <-> double. Both boxes must lie in
 * the dats' allocations (OPS_B200_ERR_ARG otherwise). Returns a halo handle. */
int ops_b200_decl_halo(int from, int to, const int *iter_size, const int *from_base, const int *to_base,
                       const int *from_dir, const int *to_dir);
/* ops_decl_halo_group (ops_lib_core.h:902). Returns a group handle. */
int ops_b200_decl_halo_group(int nhalos, const int *halos);
/* ops_halo_transfer (ops_lib_core.h:911, ops_device_singlenode_common.cpp:262):
 * flushes queued loops, then copies every halo of the group (one kernel for
 * independent halos, else one per halo in declaration order). */
int ops_b200_halo_transfer(int group);
/* ops_timers (ops/c/src/core/ops_dummy_singlenode.cpp:901): process CPU
 * seconds and monotonic wall-clock seconds. */
int ops_b200_timers(double *cpu, double *et);

/* ops_decl_const / ops_update_const (ops/c/include/ops_lib_core.h:947,971):
 * flushes queued loops, then updates every kernel constant of that name.
 * "<app>/<name>" (app = the kernels' prefix: laplace2d, cloverleaf,
 * cloverleaf3d, tealeaf) updates that app's constant only; a bare name of a
 * struct type whose layout differs between apps (field, grid, states) is
 * rejected with OPS_B200_ERR_ARG, since its size would be ambiguous. */
int ops_b200_decl_const(const char *name, int dim, const char *type, const void *data);
int ops_b200_update_const(const char *name, int dim, const char *type, const void *data);

/* One loop argument (ops_arg, ops/c/include/ops_lib_core.h:509). */
typedef struct ops_b200_arg {
  int argtype;      /* OPS_B200_ARG_*                                      */
  int dat;          /* DAT: dat handle                                     */
  int stencil;      /* DAT: stencil handle                                 */
  int dim;          /* components (DAT), elements (GBL), width (REDUCE)    */
  int acc;          /* OPS_B200_READ ... OPS_B200_MAX                      */
  int opt;          /* DAT: 1 active, 0 disabled (ops_arg_dat_opt)         */
  int reduction;    /* REDUCE: reduction handle                            */
  int elem_size;    /* GBL: bytes per element                              */
  const void *gbl;  /* GBL: payload, copied when the loop is queued        */
} ops_b200_arg;

/* ops_par_loop (ops/c/include/ops_seq_v2.h:312, queued like
 * create_kerneldesc_and_enque, ops/c/src/core/ops_lazy.cpp:1403). `kernel`
 * names a registered sm_100a loop kernel ("<app>/<kernel>", e.g.
 * "laplace2d/apply_stencil"); range has 2*dim entries {begin, end, ...}. */
int ops_b200_par_loop(const char *kernel, const char *name, int block, int dim, const int *range, int nargs,
                      const ops_b200_arg *args);
/* 1 if a loop kernel of that name is registered, else 0. */
int ops_b200_has_kernel(const char *kernel);

/* ops_execute (ops/c/src/core/ops_lazy.cpp:1248): run all queued loops. */
int ops_b200_execute(void);

/* ops_reduction_result (ops/c/src/core/ops_lib_core.cpp:1143): flushes the
 * queue and copies the handle's value (size bytes) to `out`. */
int ops_b200_reduction_result(int handle, void *out);

/* ops_dat_set_data / ops_dat_fetch_data
 * (ops/c/src/core/ops_dummy_singlenode.cpp:737-808): the full extent
 * (halos included), x fastest; `bytes` must equal that extent. On a block
 * partitioned across ranks (ops_b200_partition) they cover the rank's owned
 * part, the extents ops_b200_dat_get_extents reports. */
int ops_b200_dat_set_data(int dat, const void *data, size_t bytes);
int ops_b200_dat_fetch_data(int dat, void *data, size_t bytes);
/* ops_dat_get_extents: disp/size of the full extent (dims entries each);
 * on a partitioned block, of the rank's owned part, disp counted from the
 * dat's first point (ops/c/src/mpi/ops_mpi_rt_support.cpp:2216-2225). */
int ops_b200_dat_get_extents(int dat, int *disp, int *size);
/* ops_dat_get_raw_pointer / ops_dat_release_raw_data
 * (ops/c/src/core/ops_dummy_singlenode.cpp:662-735). Returns a pointer to
 * logical index 0 in the requested memory space; stride[0..2] receives the
 * x pitch and the y/z extents in elements. */
int ops_b200_dat_get_raw_pointer(int dat, int memspace, void **ptr, int *stride);
int ops_b200_dat_release_raw_data(int dat, int acc);

/* Runtime options: "graphs" (CUDA-graph replay of repeated flushes, default
 * 1), "fusion" (copy elision and chain kernels, default 1), "tiling"
 * (loop-chain fusion: runs of queued 2D loops executed as one kernel over
 * shared-memory tiles, default 1, needs "fusion"; the counterpart of the
 * reference's lazy tiling, ops/c/src/core/ops_lazy.cpp:380-1173) and
 * "lists" (consecutive independent loops of one kernel, e.g. over the
 * blocks of a multi-block application, launched as one kernel over a work
 * list of their uneven domains, default 1, needs "fusion").
 * "tile_candidate": -1 (default) lets the autotuner pick each fused chain's
 * tile shape and staging (or no fusion) by timing; 0..9 runs every chain
 * that fits with that one candidate (tile shape index / 2 of 64x8, 128x8,
 * 64x16, 128x16, 32x16; odd: read-only dats staged in shared memory), for
 * parity tests and profiling of the fused kernels.
 * "trid_warp": x sweeps of the batched tridiagonal solver with lines of at
 * most 256 rows run on the warp-per-lines kernel (-1, default, or 1) or on
 * the shared-memory tile kernel (0).
 * "fcg_chunks": the flexible-CG heat solves with the learned or the Jacobi
 * preconditioner replay their iterations from CUDA graphs in chunks with the
 * stopping and restart tests on the device (1, default) or run the host loop,
 * one round trip per iteration (0); both give the same iterates. */
int ops_b200_set_option(const char *name, int value);
/* Counters since the last reset: kernels launched by this library, CUDA
 * graphs launched, loops queued. */
int ops_b200_counters(long long *kernels, long long *graphs, long long *loops);
/* Loops dropped since ops_b200_init because an identical loop with unchanged
 * inputs and outputs was already queued in the same flush (no reference
 * counterpart; disabled with the "fusion" option). */
int ops_b200_loops_skipped(long long *skipped);
int ops_b200_reset_counters(void);
/* Loop-chain fusion since the last counter reset: fused kernels launched,
 * loops they replaced, and the compulsory HBM bytes of the fused kernels
 * (each dat's points read and written once per chain) against those of the
 * replaced loops run one by one. No reference counterpart. */
int ops_b200_fusion_stats(long long *chains, long long *loops, double *fused_bytes, double *loop_bytes);
/* Dat storage that the app drivers give back when they return is kept for
 * the next dats of the same size (no cudaFree/cudaMalloc of gigabytes per
 * call). This frees the kept blocks now (they are also freed and the
 * allocation retried when a dat allocation runs out of device memory) and
 * stores the bytes given back in *freed (may be NULL). No reference
 * counterpart. */
int ops_b200_release_spare_storage(long long *freed);

/* ---- Decomposition across processes (one process per GPU) ----------------
 * The reference's MPI backend (ops/c/src/mpi/): ops_partition splits every
 * block across the ranks (ops_mpi_partition.cpp:84-256, ops_decomp :257),
 * loops run over their rank's part, ops_halo_exchanges brings in the
 * neighbours' rows a stencil reads (ops_mpi_rt_support.cpp:836) and
 * reductions combine across ranks (:1271-1307). Here each block of 2 or 3
 * dimensions is split into slabs along its outermost dimension (y in 2D, z
 * in 3D) by the reference's integer division of its extent; dats of extent
 * 1 along it are replicated. Loop indices stay global. Reductions combine
 * in rank order (reproducible sums). Every rank must make the same calls in
 * the same order, as with MPI. */

/* One transfer of a host-transport exchange: send_bytes from `send` to rank
 * `peer`, and recv_bytes from `peer` into `recv` (host memory). */
typedef struct ops_b200_msg {
  int peer;
  const void *send;
  size_t send_bytes;
  void *recv;
  size_t recv_bytes;
} ops_b200_msg;
/* Host transport callbacks (return 0 on success): `exchange` completes all n
 * transfers before it returns (a rank's sends and receives may pair with
 * one another, so post them together); `allgather` stores every rank's
 * `bytes` from `send` in rank order at `recv`. */
typedef int (*ops_b200_exchange_fn)(void *ctx, const ops_b200_msg *msgs, int n);
typedef int (*ops_b200_allgather_fn)(void *ctx, const void *send, size_t bytes, void *recv);
/* The transport is set before ops_b200_partition (may precede ops_b200_init).
 * Host: the runtime flushes its queue at an exchange and stages the rows
 * through pinned memory (any transport: gloo, sockets, MPI). */
int ops_b200_set_transport_host(int nranks, int rank, ops_b200_exchange_fn exchange, ops_b200_allgather_fn allgather,
                                void *ctx);
/* NCCL (after ops_b200_init, on the runtime's device): exchanges become
 * ncclSend/ncclRecv on the runtime stream, queued and graph-captured with
 * the loops. Rank 0 makes the 128-byte id, every rank passes it. */
int ops_b200_nccl_unique_id(void *id128);
int ops_b200_set_transport_nccl(const void *id128, int nranks, int rank);
/* ops_partition (ops/c/include/ops_lib_core.h: ops_partition(const char*)):
 * partitions the blocks declared since the last call; a no-op with one rank
 * or no transport, as in the reference's single-process backends. */
int ops_b200_partition(const char *routine);
/* This process's rank and the number of ranks (1, 0 without a transport),
 * and the halo exchanges made since ops_b200_init. */
int ops_b200_rank_info(int *rank, int *nranks, long long *exchanges);
/* A block's slab on this rank: split dimension (-1: not split), the block's
 * extent along it, the owned interior [lo, hi) and the halo depth. */
int ops_b200_block_slab(int block, int *split_dim, int *extent, int *lo, int *hi, int *halo);
/* The slab arithmetic alone (no runtime, no GPU): rank `rank` of `nranks`
 * owns [lo, hi) of `extent` (ops_partition_blocks' integer division), and a
 * dat spanning [gstart, gend) along the split keeps [win_lo, win_hi) of which
 * it owns [own_lo, own_hi), with `halo` rows of each neighbour. */
int ops_b200_slab_window(int extent, int nranks, int rank, int halo, int gstart, int gend, int *lo, int *hi,
                         int *own_lo, int *own_hi, int *win_lo, int *win_hi);
/* Exercises the host transport without a GPU: each rank sends a pattern to
 * its neighbours and gathers every rank's id; returns 0 when all arrived. */
int ops_b200_transport_selftest(void);

/* Per-kernel device timing: while enabled, every launch is bracketed by CUDA
 * events on the runtime stream (graph replay is bypassed). Query by kernel
 * name ("laplace2d/apply_stencil", a chain rule name, ...): launches and total
 * milliseconds since the last clear. */
int ops_b200_set_kernel_timing(int on);
int ops_b200_kernel_time(const char *kernel, long long *launches, double *total_ms);
int ops_b200_clear_kernel_timing(void);
/* All timed kernels: up to `max` entries of name (NUL-terminated, at most 95
 * characters), launches, total milliseconds and total compulsory bytes
 * (each dat argument's points once; read-write twice). Returns the count. */
typedef struct ops_b200_kernel_stat {
  char name[96];
  long long launches;
  double total_ms;
  double alg_bytes;
} ops_b200_kernel_stat;
int ops_b200_kernel_stats(ops_b200_kernel_stat *out, int max);

/* ---- apps ----------------------------------------------------------------
 * Reference app drivers restated in C++ on the runtime above; they issue the
 * same sequence of loops as the reference drivers, ops_partition included
 * at the reference's point. With a transport of several ranks set, every
 * rank calls the driver with the same deck; outputs are then the rank's
 * owned part (Laplace: its rows of field_out; dumps: owned part per dat)
 * and reductions are global.
 *
 * Laplace Jacobi (apps/c/laplace2d_tutorial/step7/laplace2d.cpp:41-124):
 * `field_in` is A's full extent ((imax+2)*(jmax+2) doubles, x fastest, halo
 * ring = boundary values); `warmup` + `iters` fixed iterations of
 * apply_stencil + max reduction + copy. Outputs (each may be NULL): final A
 * extent, the max |delta| of each of the `warmup + iters` iterations, and the
 * device seconds (CUDA events) of the last `iters` iterations. */
int ops_b200_app_laplace2d(int imax, int jmax, int warmup, int iters, const double *field_in, double *field_out,
                           double *err_per_iter, double *device_seconds);

/* CloverLeaf 2D hydro (apps/c/CloverLeaf/clover_leaf.cpp:161-214). The deck
 * holds the values the reference reads from clover.in
 * (apps/c/CloverLeaf/read_input.cpp:36-276). */
typedef struct ops_b200_clover_state {
  double density, energy, xvel, yvel;
  int geometry;                           /* 1 rectangle, 2 circle, 3 point    */
  double xmin, xmax, ymin, ymax, radius;
} ops_b200_clover_state;

typedef struct ops_b200_clover_deck {
  int x_cells, y_cells;
  double xmin, ymin, xmax, ymax;
  double initial_timestep, timestep_rise, max_timestep, end_time;
  int end_step, summary_frequency;
  int number_of_states;                   /* 1..16; state 0 is the background */
  ops_b200_clover_state states[16];
} ops_b200_clover_deck;

/* Runs the deck to completion. Every field summary (the set-up one, one per
 * summary_frequency steps and the final one) is written to `summaries` as 8
 * doubles {step, time, volume, mass, internal energy, kinetic energy,
 * pressure sum, dt} (up to max_summaries rows; *n_summaries gets the count).
 * device_seconds: CUDA-event time of the cycles after the first
 * `warmup_steps`. dump_dir (may be NULL): every dat's full extent is written
 * to <dump_dir>/<name>.bin at the end. */
int ops_b200_app_cloverleaf(const ops_b200_clover_deck *deck, int warmup_steps, double *summaries,
                            int max_summaries, int *n_summaries, double *device_seconds, const char *dump_dir);

/* CloverLeaf 3D hydro (apps/c/CloverLeaf_3D/clover_leaf.cpp:133-213): the
 * clover.in values of the 3D app (read_input.cpp:37-276; the reference's
 * defaults are timestep_rise 1.05, max_timestep 1.0, end_time 10.0). */
typedef struct ops_b200_clover3d_state {
  double density, energy, xvel, yvel, zvel;
  int geometry;                           /* 1 cuboid, 2 sphere, 3 point       */
  double xmin, xmax, ymin, ymax, zmin, zmax, radius;
} ops_b200_clover3d_state;

typedef struct ops_b200_clover3d_deck {
  int x_cells, y_cells, z_cells;
  double xmin, ymin, zmin, xmax, ymax, zmax;
  double initial_timestep, timestep_rise, max_timestep, end_time;
  int end_step, summary_frequency;
  int number_of_states;                   /* 1..16; state 0 is the background */
  ops_b200_clover3d_state states[16];
} ops_b200_clover3d_deck;

/* Runs the 3D deck to completion; outputs as ops_b200_app_cloverleaf (8
 * doubles per field summary, kinetic energy over the eight nodes of a cell). */
int ops_b200_app_cloverleaf3d(const ops_b200_clover3d_deck *deck, int warmup_steps, double *summaries,
                              int max_summaries, int *n_summaries, double *device_seconds, const char *dump_dir);

/* TeaLeaf 2D implicit heat conduction (apps/c/TeaLeaf/diffuse.cpp:78-148,
 * tea_solve.cpp:37-418). The deck holds the tea.in values the reference
 * reads (apps/c/TeaLeaf/read_input.cpp:70-378); states use the CloverLeaf
 * state record (velocities ignored). solver: 0 Jacobi, 1 CG, 2 Chebyshev
 * (tl_use_chebyshev), 3 polynomially preconditioned CG (tl_use_ppcg);
 * preconditioner: 0 none, 1 Jacobi diagonal (jac_diag); coefficient:
 * 1 conductivity = density, 2 reciprocal density. Solvers 2 and 3 start
 * with CG and switch once the error is <= ch_cg_epslim after at least
 * ch_cg_presteps iterations (tea_solve.cpp:146-160; the reference defaults
 * are 25 and 1.0); ppcg_inner_steps is the polynomial degree, -1 for the
 * reference's guess 4 * (int)sqrt(sqrt(x_cells * y_cells))
 * (read_input.cpp:351-354). These three are read as given: a deck zeroed
 * by the caller switches at once and never by error.
 * Beyond tea.in (no reference counterpart): fused = 1 runs each CG solve as
 * the device-resident three-kernel iteration (alpha, beta and the stop test
 * stay on the GPU; same per-cell arithmetic and stopping rule as the loop
 * chain, which fused = 0 keeps); true_residual_stop = 1 (with fused) stops on
 * ||r|| < eps * ||r0|| instead of TeaLeaf's sqrt|r.z|; mixed = 1 (with fused)
 * runs the iteration in FP32 under FP64 reliable updates (the FP32 residual
 * is replaced by u0 - A u computed in FP64 each time it has fallen by
 * reliable_delta, search direction kept) and stops when the FP64 residual
 * ||u0 - A u|| < eps * ||r0||. Fused solves need reflective_boundary = 0. */
typedef struct ops_b200_tea_deck {
  int x_cells, y_cells;
  double xmin, ymin, xmax, ymax;
  double initial_timestep, end_time;
  int end_step, summary_frequency;
  int max_iters;
  double eps;
  int coefficient, preconditioner, solver, reflective_boundary, check_result;
  int number_of_states;                   /* 1..24; state 0 is the background */
  ops_b200_clover_state states[24];
  int fused, mixed, true_residual_stop;
  double reliable_delta;
  int ch_cg_presteps;                     /* tl_ch_cg_presteps */
  double ch_cg_epslim;                    /* tl_ch_cg_epslim */
  int ppcg_inner_steps;                   /* tl_ppcg_inner_steps */
} ops_b200_tea_deck;

/* Runs the deck. summaries: 6 doubles per field summary {step, time, volume,
 * mass, internal energy, temperature}; solves: OPS_B200_TEA_SOLVE_COLS
 * doubles per timestep solve {iterations (as tea_solve.cpp:386 prints them),
 * initial residual, final stopping quantity / initial residual, exact residual
 * ratio (tl_check_result) or -1, true FP64 residual ratio ||u0 - A u|| / ||r0||
 * at exit or -1 (fused solves compute it), reliable updates (mixed) or 0,
 * device seconds of the solve (coefficient set-up through finalise),
 * PPCG inner iterations (tea_solve.cpp:389-392) or 0, the iteration n at
 * which Chebyshev or PPCG took over or -1, the eigenvalue bounds in use
 * (estimate scaled by 0.95 and 1.05) or 0, Chebyshev's estimated iteration
 * count est_itc or -1}. dump_dir as for CloverLeaf. */
#define OPS_B200_TEA_SOLVE_COLS 12
int ops_b200_app_tealeaf(const ops_b200_tea_deck *deck, double *summaries, int max_summaries, int *n_summaries,
                         double *solves, int max_solves, int *n_solves, double *device_seconds, const char *dump_dir);

/* ---- batched tridiagonal solves ------------------------------------------
 * ops_tridMultiDimBatch / ops_tridMultiDimBatch_Inc
 * (ops/c/include/ops_tridiag.h, ops/c/src/tridiag/ops_tridiag.cpp:78-249):
 * solve a_i x_{i-1} + b_i x_i + c_i x_{i+1} = d_i along dimension `solvedim`
 * for every line of `range` (2*ndim entries). The plain form overwrites d
 * with x; _Inc adds x to u and leaves d untouched. a, b, c, d (and u) are dat
 * handles of one type ("double" or "float") and one shape. The reference's
 * ops_tridsolver_params only steer the MPI strategies and are not needed on
 * one GPU. Queued loops are flushed first. */
int ops_b200_tridMultiDimBatch(int ndim, int solvedim, const int *range, int a, int b, int c, int d);
int ops_b200_tridMultiDimBatch_Inc(int ndim, int solvedim, const int *range, int a, int b, int c, int d, int u);

/* ops_tridsolver_params (ops/c/include/ops_tridiag.h:45-72): the strategy
 * and tuning values of Tridsolver's multi-process solves, held in a plain
 * struct instead of the reference's class. _init stands for both
 * constructors (strategy -1 = the reference's default, GATHER_SCATTER = 0;
 * JACOBI 2, PCR 3, LATENCY_HIDING_INTERLEAVED 4, LATENCY_HIDING_TWO_STEP 5);
 * the setters mirror set_jacobi_params, set_batch_size, set_cuda_opts and
 * set_cuda_sync and only record their values: as in the reference's
 * single-process backends (ops/c/src/tridiag/ops_tridiag.cpp:48-76), nothing
 * on one GPU reads them. Invalid values are OPS_B200_ERR_ARG. */
typedef struct ops_b200_tridsolver_params {
  int block, strategy;
  double jacobi_rtol, jacobi_atol;
  int jacobi_maxiter, batch_size;
  int cuda_opts[3];
  int cuda_sync;
} ops_b200_tridsolver_params;
int ops_b200_tridsolver_params_init(ops_b200_tridsolver_params *p, int block, int strategy);
int ops_b200_tridsolver_params_set_jacobi_params(ops_b200_tridsolver_params *p, double rtol, double atol,
                                                 int maxiter);
int ops_b200_tridsolver_params_set_batch_size(ops_b200_tridsolver_params *p, int batch_size);
int ops_b200_tridsolver_params_set_cuda_opts(ops_b200_tridsolver_params *p, int opt_x, int opt_y, int opt_z);
int ops_b200_tridsolver_params_set_cuda_sync(ops_b200_tridsolver_params *p, int sync);

/* One strided system set, as Tridsolver's trid{D,S}mtsvStridedBatch[Inc]
 * takes it (call sites ops/c/src/tridiag/ops_tridiag.cpp:126,140,219,236):
 * device pointers to the first solved element, the solved extents `dims`
 * and the allocated extents `pads` (element (i,j,k) at
 * i + j*pads[0] + k*pads[0]*pads[1]); u != NULL selects the Inc form. */
typedef struct ops_b200_trid_system {
  const void *a, *b, *c;
  void *d, *u;
  int ndim;
  int dims[3];
  int pads[3];
} ops_b200_trid_system;

/* Solves all lines along `solvedim` of `nsys` system sets, of any shapes, in
 * one launch (elem_size 8 = double, 4 = float) on `stream` (cudaStream_t,
 * NULL = default stream). Lines along x (contiguous) run the partition
 * method in shared memory, up to 512 points; lines along y/z (strided,
 * neighbouring lines contiguous) run Thomas per line, any length, with a
 * c'/d' scratch array of 2 x (unknowns) elements that the library keeps and
 * grows. The work lists and that scratch are shared by all calls: calls on
 * different streams must not overlap. */
int ops_b200_trid_batch(int elem_size, int solvedim, int nsys, const ops_b200_trid_system *systems, void *stream);

/* ---- allocation-free sweep ----------------------------------------------
 * No counterpart in the reference: an extra entry point for callers that
 * cannot allocate device memory where they need a sweep (inside another
 * framework's memory pool or arena, inside a stream capture that must not
 * gain allocation nodes, or in latency-critical loops).
 *
 * One Jacobi sweep of the Laplace 5-point stencil, the arithmetic of loop
 * kernel "laplace2d/apply_stencil": Anew = 0.25 * (A(+1,0) + A(-1,0) +
 * A(0,-1) + A(0,+1)) over x in [0, imax), y in [0, jmax), and the maximum
 * |Anew - A| written to *max_delta. A and Anew are device pointers to
 * logical index (0,0) of fields with a one-cell halo and a row pitch of
 * `pitch` doubles (>= imax + 2); max_delta is a device pointer; stream is a
 * cudaStream_t (NULL = default stream). Nothing is allocated: the scratch is
 * a fixed ~32 KiB __device__ array that every GPU loading this library holds
 * until exit. imax and jmax above 65536 are rejected (OPS_B200_ERR_ARG).
 * All calls share that array, so calls that can overlap on the GPU race and
 * must be serialised by the caller. The first call on each device looks up
 * the array's device address; make it before any stream capture. Errors are
 * described by ops_b200_noalloc_last_error(). */
int ops_b200_laplace_sweep_noalloc(int imax, int jmax, const double *A, double *Anew, long long pitch,
                                   double *max_delta, void *stream);
const char *ops_b200_noalloc_last_error(void);

/* ---- learned preconditioner building blocks (no reference counterpart) --
 * 3x3 convolution, stride 1, zero padding 1, on the tcgen05 tensor cores:
 * x NHWC BF16 [n][h][w][cin], weights BF16 [9][cout][cin] (tap = (dy+1)*3 +
 * (dx+1)), y NHWC BF16 [n][h][w][cout], FP32 accumulation. mode 0: y =
 * relu(conv + bias); 1: y = conv + bias; 2: y = conv * (mask > 0) with mask
 * BF16 shaped like y; 3: y = conv. (cin, cout) in {(16,16), (16,32), (32,16),
 * (32,32), (32,64), (64,32), (64,64)}; pointers 16-byte aligned. Synchronous
 * on `stream` (a cudaStream_t, NULL = default); OPS_B200_ERR_TIMEOUT if a
 * pipeline wait inside the kernel expired. */
int ops_b200_conv3x3_bf16(const void *x, const void *w, const float *bias, const void *mask, void *y, int n, int h,
                          int wd, int cin, int cout, int mode, void *stream);

/* ---- heat solves on caller-owned device fields (no reference counterpart)
 * The TeaLeaf operator A u = (1 + rx (Kx + Kx_e) + ry (Ky + Ky_n)) u - ...
 * (apps/c/TeaLeaf/tea_leaf_common_kernels.h) on an nx x ny interior. Every
 * pointer addresses the first interior cell of an FP64 field with a one-cell
 * ring (index -1 .. n), row pitch `pitch` elements; Kx and Ky are the face
 * coefficients TeaLeaf's tea_leaf_common_init_Kx_Ky_kernel produces (zero on
 * the domain boundary). u holds the initial guess and receives the solution.
 * The solve stops when ||u0 - A u|| < eps ||r0|| (method 0: TeaLeaf's
 * sqrt|r.z| test) or after max_iters iterations. */
typedef struct ops_b200_heat_system {
  int nx, ny;
  long long pitch;
  const double *Kx, *Ky, *u0;
  double *u;
  double rx, ry;
} ops_b200_heat_system;

typedef struct ops_b200_heat_stats {
  int iterations;          /* CG iterations (method 0: as TeaLeaf prints them) */
  int updates;             /* reliable updates (method 2) */
  int converged;
  int fallbacks;           /* switches to the fallback preconditioner (methods 3, 5, 6) */
  double initial_residual; /* ||u0 - A u|| at entry */
  double final_residual;   /* ||u0 - A u|| at exit, FP64 */
  double seconds;          /* device time of the solve */
  long long launches;      /* kernels launched by the solve */
} ops_b200_heat_stats;

#define OPS_B200_HEAT_PCG 0          /* FP64 Jacobi-PCG, TeaLeaf's stopping rule */
#define OPS_B200_HEAT_PCG_TRUE 1     /* FP64 Jacobi-PCG, stop on ||r|| < eps ||r0|| */
#define OPS_B200_HEAT_MIXED 2        /* FP32 Jacobi-PCG under FP64 reliable updates */
#define OPS_B200_HEAT_FCG_LEARNED 3  /* flexible CG, learned preconditioner `net`, Jacobi fallback */
#define OPS_B200_HEAT_FCG_JACOBI 4   /* the same flexible CG with Jacobi (no network) */
#define OPS_B200_HEAT_FCG_MG 5       /* the same flexible CG, one native multigrid V-cycle per iteration */
#define OPS_B200_HEAT_FCG_LEARNED_MG 6 /* flexible CG, M(r) = V-cycle(r) + the correction of network `net`
                                          (trained on targets e - V-cycle(r)); falls back to the V-cycle */

/* Solves A u = u0. `net` names a learned preconditioner (methods 3, 6);
 * window: methods 3, 5 and 6 fall back (to Jacobi; method 6 to the V-cycle
 * alone) when ||r|| has not halved over `window` iterations (0 = only on
 * lost positive curvature). r_out (device, may be
 * NULL) receives u0 - A u at exit. Synchronous on `stream`. Not reentrant:
 * one solve at a time per process (a shared workspace is kept per size). */
int ops_b200_heat_solve(const ops_b200_heat_system *sys, int method, int net, double eps, int max_iters, int window,
                        double *r_out, ops_b200_heat_stats *stats, void *stream);

/* The 3D 7-point heat operator (the 512^3 case of the heat solve; no
 * reference counterpart: OPS TeaLeaf is 2D): A u = (1 + rx (Kx + Kx+x) +
 * ry (Ky + Ky+y) + rz (Kz + Kz+z)) u - rx (Kx+x u+x + Kx u-x) - ... with
 * face conductivities K (Kz(x,y,z) the face between z-1 and z). Pointers
 * address the first interior cell of FP64 volumes with one halo cell on
 * each side; plane == pitch * (ny + 2). Methods OPS_B200_HEAT_PCG and
 * OPS_B200_HEAT_PCG_TRUE (FP64 Jacobi-PCG, device-resident iterations) and
 * OPS_B200_HEAT_MIXED (FP32 Jacobi-PCG under FP64 reliable updates).
 * Synchronous on `stream`; not reentrant (a workspace is kept per size). */
typedef struct ops_b200_heat_system3d {
  int nx, ny, nz;
  long long pitch, plane;
  const double *Kx, *Ky, *Kz, *u0;
  double *u;
  double rx, ry, rz;
} ops_b200_heat_system3d;
int ops_b200_heat_solve3d(const ops_b200_heat_system3d *sys, int method, double eps, int max_iters,
                          ops_b200_heat_stats *stats, void *stream);

/* Native multigrid preconditioner of method 5: z = M r, one FP32 V-cycle
 * over a hierarchy of 2 x 2 aggregates (coarse mass = sum of the aggregate's,
 * coarse face weight = half the sum of the fine faces it covers, coarsening
 * down to at most 16 x 16 cells), two damped-Jacobi sweeps (omega 0.8) before
 * and after each coarse correction, 64 sweeps on the coarsest level. The
 * hierarchy is built from sys (Kx, Ky, rx, ry; u0 and u are not read); r and
 * z are device fields laid out like sys's (same pitch). *levels (may be
 * NULL) receives the number of levels. Synchronous on `stream`. */
int ops_b200_heat_mg_apply(const ops_b200_heat_system *sys, const double *r, double *z, int *levels, void *stream);

/* ---- learned multigrid preconditioner (no reference counterpart) ---------
 * A 4-level U-Net-shaped CNN (16/32/64/64 channels, 3x3 BF16 convolutions on
 * the tensor cores, FP32 accumulation) mapping a residual and the face
 * coefficients to M(r) = r / diag(A) + s * net(r / s, ...), s = rms(r);
 * trained on residual/error pairs (loss mean_n ||M(r_n) - e_n||^2 / ||e_n||^2)
 * by the library's own forward and backward kernels with Adam. A batch is n
 * fields of h x w interior cells (multiples of 8) laid out like
 * ops_b200_heat_system, image n starting `image` elements after image 0. */
typedef struct ops_b200_heat_batch {
  int n, h, w;
  long long pitch, image;
  const double *r, *Kx, *Ky;
  double rx, ry;
} ops_b200_heat_batch;

int ops_b200_lmg_create(unsigned long long seed);   /* returns a handle */
int ops_b200_lmg_destroy(int net);
int ops_b200_lmg_num_params(void);
/* FP32 parameters: per conv layer W [9][cout][cin] then b [cout] (layers
 * C0, C1a, C1b, C2a, C2b, C3a, C3b, C2u, C1u, C0u), then wout [16], bout. */
int ops_b200_lmg_get_params(int net, float *host);
int ops_b200_lmg_set_params(int net, const float *host);   /* also resets Adam */
int ops_b200_lmg_get_grads(int net, float *host);          /* of the last train step */
/* out (device, batch layout) = M(r). Synchronous on `stream`. */
int ops_b200_lmg_apply(int net, const ops_b200_heat_batch *b, double *out, void *stream);
/* Forward + backward on a batch with targets e (device, batch layout); one
 * Adam step when lr > 0; *loss receives the batch loss before the step.
 * loss_kind 0: mean_n ||M(r) - e||^2 / ||e||^2; 1: the same ratio in the
 * A-norm, d.Ad / e.Ae with d = M(r) - e (what CG convergence depends on). */
int ops_b200_lmg_train_step(int net, const ops_b200_heat_batch *b, const double *e, int loss_kind, double lr,
                            double *loss, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* OPS_B200_H */
