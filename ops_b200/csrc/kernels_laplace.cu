// Laplace (Jacobi relaxation) loop kernels.
//
// Point kernels restate apps/c/laplace2d_tutorial/step7/laplace_kernels.h
// (set_zero :6, copy :10, left_bndcon :14, right_bndcon :18,
// apply_stencil :22) with the same operation order; compiled with
// --fmad=false every cell update is bit-identical to the reference's CPU
// build. The boundary kernels call the device sin/exp, which can differ from
// the host libm in the last bit; seeded runs set their boundary from the host.
#include <cstddef>

#include "runtime.h"

namespace opsb {
namespace laplace {

struct Consts {
  int imax, jmax;
  double pi;
};
__constant__ Consts c_lap;

struct set_zero {
  static constexpr const char *kname = "laplace2d/set_zero";
  __device__ void operator()(ACC2<double> &A) const { A(0, 0) = 0.0; }
};

struct copy {
  static constexpr const char *kname = "laplace2d/copy";
  // Pure copy: dst = arg 0, src = arg 1 (used by the runtime's copy elision).
  static constexpr int copy_dst = 0, copy_src = 1;
  __device__ void operator()(ACC2<double> &A, const ACC2<double> &Anew) const { A(0, 0) = Anew(0, 0); }
};

struct left_bndcon {
  static constexpr const char *kname = "laplace2d/left_bndcon";
  __device__ void operator()(ACC2<double> &A, const IDX &idx) const {
    A(0, 0) = sin(c_lap.pi * (idx[1] + 1) / (c_lap.jmax + 1));
  }
};

struct right_bndcon {
  static constexpr const char *kname = "laplace2d/right_bndcon";
  __device__ void operator()(ACC2<double> &A, const IDX &idx) const {
    A(0, 0) = sin(c_lap.pi * (idx[1] + 1) / (c_lap.jmax + 1)) * exp(-c_lap.pi);
  }
};

struct apply_stencil {
  static constexpr const char *kname = "laplace2d/apply_stencil";
  __device__ void operator()(const ACC2<double> &A, ACC2<double> &Anew, RED<double> &error) const {
    Anew(0, 0) = 0.25f * (A(1, 0) + A(-1, 0) + A(0, -1) + A(0, 1));
    *error = fmax(*error, fabs(Anew(0, 0) - A(0, 0)));
  }
};

OPSB_REGISTER_LOOP(set_zero);
OPSB_REGISTER_LOOP(copy);
OPSB_REGISTER_LOOP(left_bndcon);
OPSB_REGISTER_LOOP(right_bndcon);
OPSB_REGISTER_LOOP(apply_stencil);

struct ConstReg {
  ConstReg() {
    Runtime::register_const("laplace2d/imax", &c_lap, offsetof(Consts, imax), sizeof(int));
    Runtime::register_const("laplace2d/jmax", &c_lap, offsetof(Consts, jmax), sizeof(int));
    Runtime::register_const("laplace2d/pi", &c_lap, offsetof(Consts, pi), sizeof(double));
  }
};
static ConstReg const_reg;

}  // namespace laplace
}  // namespace opsb

namespace opsb {
// Typed par_loop call sites used by the C++ Laplace driver (apps_laplace.cpp).
void laplace_par_loop_apply(int block, const int *range, int dA, int dAnew, int s5, int s0, int h_err) {
  par_loop<laplace::apply_stencil>("apply stencil", block, 2, range,
                                   {arg_dat(dA, 1, s5, ACC_READ), arg_dat(dAnew, 1, s0, ACC_WRITE),
                                    arg_reduce(h_err, 1, ACC_MAX)});
}
void laplace_par_loop_copy(int block, const int *range, int dA, int dAnew, int s0) {
  par_loop<laplace::copy>("copy", block, 2, range, {arg_dat(dA, 1, s0, ACC_WRITE), arg_dat(dAnew, 1, s0, ACC_READ)});
}
}  // namespace opsb
