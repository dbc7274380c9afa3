// Native multigrid preconditioner for the TeaLeaf 2D heat operator
// (A u = (1 + rx (Kx_w + Kx_e) + ry (Ky_s + Ky_n)) u - rx (Kx_e u_e + Kx_w u_w)
//        - ry (Ky_n u_n + Ky_s u_s), tea_leaf_common_kernels.h), the
// non-learned counterpart of the learned U-Net preconditioner: one V-cycle
// z = M r per flexible-CG iteration.
//
// Hierarchy (built by `setup`, FP32):
//  - level 0 is the operator itself, with face weights ax = rx Kx, ay = ry Ky
//    rounded to FP32 and unit mass;
//  - a coarse cell aggregates 2 x 2 cells of the level below (a lone row or
//    column at an odd edge aggregates 1 x 2 or 2 x 1); its mass is the sum of
//    their masses and each coarse face weight is `kFaceScale` (1/2) times the
//    sum of the fine face weights it covers. The Galerkin operator of
//    piecewise-constant aggregation (scale 1) makes the coarse faces twice as
//    stiff as a rediscretisation at 2h; halving them restores the
//    rediscretised scaling (on the seeded 1024^2 heat problem, 24 flexible-CG
//    iterations to 1e-10 with the Galerkin faces, 11 with the halved ones);
//  - coarsening stops when both sides are at most `kCoarsest` (16) cells; that
//    level is solved by `kCoarseSweeps` damped-Jacobi sweeps in one CTA.
//
// Cycle (per level above the coarsest, nu = `kSweeps` = 2, omega = 0.8):
//    z = omega r / c; nu - 1 more damped-Jacobi sweeps;
//    r_c = R (r - A z) (sum over the aggregate); e = cycle(level + 1, r_c);
//    z += P e (injection) fused into the first of nu post-sweeps.
// Pre- and post-smoothing match, so the cycle is a symmetric operator up to
// FP32 rounding; the outer flexible CG (FP64) tolerates the rounding.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace opsb {
namespace heat {

class Multigrid {
 public:
  static constexpr int kCoarsest = 16;
  static constexpr int kSweeps = 2;
  static constexpr int kCoarseSweeps = 64;
  static constexpr float kOmega = 0.8f;
  static constexpr float kFaceScale = 0.5f;

  Multigrid() = default;
  ~Multigrid();
  Multigrid(const Multigrid &) = delete;
  Multigrid &operator=(const Multigrid &) = delete;

  // Builds the hierarchy for the operator on an nx x ny interior whose FP64
  // fields share `pitch` (Kx, Ky address the first interior cell; the face
  // weights read are Kx[y pitch + x] for x in [0, nx] and Ky[y pitch + x]
  // for y in [0, ny]). Storage is kept while the shape stays the same.
  void setup(int nx, int ny, long long pitch, const double *Kx, const double *Ky, double rx, double ry,
             cudaStream_t s);
  // z = M r on the interior (FP64, `pitch` of the setup); returns the kernels
  // launched. The cycle's launches are captured into a CUDA graph on first
  // use for a given (r, z, stream) and replayed from it afterwards; the
  // graph reads the hierarchy through its pointers, so a later setup of the
  // same shape (new coefficients, same storage) keeps it valid.
  long long apply(const double *r, double *z, cudaStream_t s);
  int levels() const { return (int)lv_.size(); }

 private:
  long long enqueue(const double *r, double *z, cudaStream_t s);
  void drop_graph();
  cudaGraphExec_t exec_ = nullptr;
  const double *g_r_ = nullptr;
  double *g_z_ = nullptr;
  cudaStream_t g_s_ = nullptr;
  long long g_n_ = 0;
  struct Level {
    int nx = 0, ny = 0;
    long long pitch = 0;  // elements; rows of the face arrays hold nx + 1
    float *m = nullptr;   // mass (nullptr on level 0: unit mass)
    float *ax = nullptr, *ay = nullptr;
    float *r = nullptr, *z0 = nullptr, *z1 = nullptr;
  };
  void release();
  std::vector<Level> lv_;
  float *buf_ = nullptr;
  size_t buf_elems_ = 0;
  long long fpitch_ = 0;  // pitch of the FP64 fields
};

}  // namespace heat
}  // namespace opsb
