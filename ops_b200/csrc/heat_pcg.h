// Device-resident Jacobi-preconditioned CG for the TeaLeaf 2D heat operator
// (apps/c/TeaLeaf/tea_solve.cpp:139-356 with tea_leaf_cg.cpp:53-214): the
// scalars alpha, beta and the stopping test live in device memory, so an
// iteration is three kernel launches and no host round trip; iterations are
// replayed from a CUDA graph in chunks and the host polls one chunk behind.
//
// Two precisions:
//  - pcg_fp64: the reference's FP64 iteration, cell for cell (w = A p with
//    pw = p.w; u += alpha p, r -= alpha w, z = Mi r with rz = r.z; p = beta p + z)
//    and TeaLeaf's stopping rule sqrt|rz| < eps * ||r0||.
//    With true_stop the test is ||r|| < eps * ||r0|| on the recursive residual.
//  - pcg_mixed: the same iteration in FP32 (r, p, w, z and the correction e,
//    with FP32 copies of Kx, Ky, Mi) under FP64 reliable updates (Sleijpen and
//    van der Vorst 1996): whenever the recursive sqrt(r.z) has fallen by
//    `delta` since the last update, or its estimate says converged, e is added
//    to u in FP64, r = u0 - A u is recomputed in FP64 and replaces the FP32
//    residual, and the search direction is kept. The solve stops when that
//    FP64 residual ||u0 - A u|| < eps * ||r0||.
//  - fcg: flexible CG (Notay 2000, one-step truncation) with a caller-supplied
//    preconditioner z = M(r) (the learned one), alpha = p.r / p.w,
//    beta = -z.w / p.w; it falls back to Jacobi and restarts the recursion
//    when p.w <= 0 or when ||r|| has not halved over `window` iterations.
#pragma once
#include <cuda_runtime.h>

#include <functional>

namespace opsb {
namespace heat {

// Interior of one TeaLeaf chunk: every pointer addresses the first interior
// cell of an FP64 field with one halo cell on each side; all share `pitch`.
struct Field2D {
  int nx = 0, ny = 0;
  long long pitch = 0;
  const double *Kx = nullptr, *Ky = nullptr, *u0 = nullptr;
  double *u = nullptr, *r = nullptr, *w = nullptr, *p = nullptr, *z = nullptr, *Mi = nullptr;
};

// The 3D 7-point operator's fields: pointers address the first interior
// cell of FP64 volumes with one halo cell on each side, x fastest, `pitch`
// elements between rows and plane == pitch * (ny + 2) between z planes. The
// solver's own fields (r, w, p, z, Mi) must be zero on every halo cell.
struct Field3D {
  int nx = 0, ny = 0, nz = 0;
  long long pitch = 0, plane = 0;
  const double *Kx = nullptr, *Ky = nullptr, *Kz = nullptr, *u0 = nullptr;
  double *u = nullptr, *r = nullptr, *w = nullptr, *p = nullptr, *z = nullptr, *Mi = nullptr;
};

struct SolveStats {
  int iterations = 0;         // as the reference reports it (n - 1 on convergence)
  int outer = 0;              // reliable updates (mixed only)
  int converged = 0;
  int fallbacks = 0;          // learned -> Jacobi switches (fcg only)
  double initial_residual = 0; // ||u0 - A u|| at entry
  double error = 0;            // the stopping quantity at exit
  double true_residual = 0;    // ||u0 - A u|| at exit, FP64
};

class Solver {
 public:
  Solver();
  ~Solver();
  Solver(const Solver &) = delete;
  Solver &operator=(const Solver &) = delete;

  void pcg_fp64(const Field2D &f, double rx, double ry, bool precond, bool true_stop, double eps, int max_iters,
                cudaStream_t s, SolveStats *st);
  void pcg_mixed(const Field2D &f, double rx, double ry, bool precond, double eps, double delta, int max_iters,
                 cudaStream_t s, SolveStats *st);
  // z = M(r) on the interior of the solve's fields; returns kernels launched.
  using Precond = std::function<long long(const double *r, double *z, cudaStream_t s)>;
  // On a restart (p.w <= 0, or no halving of ||r|| over `window`
  // iterations) the solve continues with `fallback` when one is given, else
  // with Jacobi.
  // With `chunked`, M (and the fallback) must be stream-capturable (kernel
  // launches and memsets only, after one call outside capture): iterations
  // are then replayed from CUDA graphs in chunks, with the stopping and
  // restart tests on the device and the host polling one chunk behind;
  // iteration counts and results are those of the host loop.
  void fcg(const Field2D &f, double rx, double ry, double eps, int max_iters, const Precond &M, int window,
           cudaStream_t s, SolveStats *st, const Precond *fallback = nullptr, bool chunked = false);
  // The same FP64 Jacobi-PCG for the 3D 7-point operator (stopping rule as
  // pcg_fp64: TeaLeaf's sqrt|r.z|, or ||r|| with true_stop).
  void pcg3d(const Field3D &f, double rx, double ry, double rz, bool true_stop, double eps, int max_iters,
             cudaStream_t s, SolveStats *st);
  void diag3(const Field3D &f, double rx, double ry, double rz, cudaStream_t s);
  // pcg_mixed for the 3D operator: FP32 PCG under FP64 reliable updates,
  // stopping on the FP64 ||u0 - A u|| < eps ||r0||. f.Mi must hold diag3's.
  void pcg3d_mixed(const Field3D &f, double rx, double ry, double rz, double eps, double delta, int max_iters,
                   cudaStream_t s, SolveStats *st);
  // Mi = 1 / diag(A) on the interior (tea_leaf_common_init_diag_init_kernel).
  void diag(const Field2D &f, double rx, double ry, cudaStream_t s);
  // out = u0 - A u on the interior; returns ||out||.
  double residual(const Field2D &f, double rx, double ry, double *out, cudaStream_t s);
  // Kernels launched by the last solve (each launch counted once, including
  // the no-op launches of a chunk that ran past convergence).
  long long launches() const { return launches_; }

 private:
  struct Impl;
  Impl *m_;
  long long launches_ = 0;
};

}  // namespace heat
}  // namespace opsb
