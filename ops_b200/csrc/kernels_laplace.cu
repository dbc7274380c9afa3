// Laplace (Jacobi relaxation) loop kernels.
//
// Point kernels restate apps/c/laplace2d_tutorial/step7/laplace_kernels.h
// (set_zero :6, copy :10, left_bndcon :14, right_bndcon :18,
// apply_stencil :22) with the same operation order; compiled with
// --fmad=false every cell update is bit-identical to the reference's CPU
// build. The boundary kernels call the device sin/exp, which can differ from
// the host libm in the last bit; seeded runs set their boundary from the host.
#include <algorithm>
#include <cstddef>
#include <cstdint>

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

// The Jacobi sweep with its max|delta| reduction as a column march: each
// thread owns one x and a chunk of kRows rows, walking up in y with the
// centre column's three rows (y-1, y, y+1) in registers, so a point costs
// three loads (the row above and the two x neighbours, the latter from L1)
// instead of five. Same expression and operation order as the functor.
template <int X, int R, int B>
__global__ void __launch_bounds__(X) apply_stencil_march(const __grid_constant__ LoopParams lp) {
  const ArgView &va = lp.a[0], &vn = lp.a[1], &vr = lp.a[2];
  const double *A = reinterpret_cast<const double *>(va.ptr);
  double *An = reinterpret_cast<double *>(vn.ptr);
  const long long pa = va.ay, pn = vn.ay;
  const int x = lp.start[0] + blockIdx.x * X + threadIdx.x;
  const int y0 = lp.start[1] + blockIdx.y * R;
  const int y1 = min(y0 + R, lp.end[1]);
  double err = red_identity<double>(ACC_MAX);
  if (x < lp.end[0] && y0 < y1) {
    const double *col = A + x;
    double dn = __ldg(col + (y0 - 1) * pa);
    double c = __ldg(col + y0 * pa);
    int y = y0;
    // B rows at a time: all their loads are issued before any arithmetic
    for (; y + B <= y1; y += B) {
      double up[B], r[B], l[B];
#pragma unroll
      for (int k = 0; k < B; k++) {
        up[k] = __ldg(col + (y + k + 1) * pa);
        r[k] = __ldg(col + (y + k) * pa + 1);
        l[k] = __ldg(col + (y + k) * pa - 1);
      }
#pragma unroll
      for (int k = 0; k < B; k++) {
        const double v = 0.25f * (r[k] + l[k] + dn + up[k]);  // A(1,0) + A(-1,0) + A(0,-1) + A(0,1)
        An[x + (long long)(y + k) * pn] = v;
        err = fmax(err, fabs(v - c));
        dn = c;
        c = up[k];
      }
    }
    for (; y < y1; y++) {
      const double up = __ldg(col + (y + 1) * pa);
      const double v = 0.25f * (__ldg(col + y * pa + 1) + __ldg(col + y * pa - 1) + dn + up);
      An[x + (long long)y * pn] = v;
      err = fmax(err, fabs(v - c));
      dn = c;
      c = up;
    }
  }
  // block maximum, then the last block folds the partials in block order
  __shared__ double smem[32];
  __shared__ int last;
  const int nblocks = gridDim.x * gridDim.y;
  const double b = block_reduce<double>(err, ACC_MAX, smem);
  const int bid = blockIdx.x + blockIdx.y * gridDim.x;
  if (threadIdx.x == 0) {
    reinterpret_cast<double *>(lp.red_scratch)[((size_t)vr.red_index * nblocks + bid) * OPSB_MAX_RED_DIM] = b;
    __threadfence();
    last = (atomicAdd(lp.red_counter, 1u) == (unsigned int)(nblocks - 1));
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  finish_grid_reduction<double>(vr, lp, nblocks, smem);
  if (threadIdx.x == 0) *lp.red_counter = 0u;
}

// Two columns per thread: one 16-byte load per row gives a thread its pair
// (x, x+1); x-1 and x+2 come from the neighbouring lanes by warp shuffles
// (the warp's first and last lane load theirs). Needs an even x start and
// an even pitch (16-byte aligned pairs).
template <int X, int R, int B>
__global__ void __launch_bounds__(X) apply_stencil_march2(const __grid_constant__ LoopParams lp) {
  const ArgView &va = lp.a[0], &vn = lp.a[1], &vr = lp.a[2];
  const double *A = reinterpret_cast<const double *>(va.ptr);
  double *An = reinterpret_cast<double *>(vn.ptr);
  const long long pa = va.ay, pn = vn.ay;
  const int lane = threadIdx.x & 31;
  const int x = lp.start[0] + 2 * (blockIdx.x * X + threadIdx.x);
  const int y0 = lp.start[1] + blockIdx.y * R;
  const int y1 = min(y0 + R, lp.end[1]);
  const bool in0 = x < lp.end[0], in1 = x + 1 < lp.end[0];
  const bool any = __any_sync(0xffffffffu, in0);
  double err = red_identity<double>(ACC_MAX);
  if (any && y0 < y1) {
    // a pair reads x-1 .. x+2 (all inside the allocation for an in-range
    // x: the stencil reaches one point past the range); a thread whose pair
    // starts past the range loads nothing
    auto ld2 = [&](int y) -> double2 {
      const double *p = A + x + (long long)y * pa;
      if (in1) return __ldg(reinterpret_cast<const double2 *>(p));
      double2 v;
      v.x = in0 ? __ldg(p) : 0.0;
      v.y = in0 ? __ldg(p + 1) : 0.0;
      return v;
    };
    double2 dn = ld2(y0 - 1), c = ld2(y0);
    for (int y = y0; y < y1; y += B) {
      double2 up[B];
      double lx[B], rx[B];
#pragma unroll
      for (int k = 0; k < B; k++) {
        up[k] = (y + k < y1) ? ld2(y + k + 1) : make_double2(0.0, 0.0);
        const double *row = A + x + (long long)(y + k) * pa;
        lx[k] = (lane == 0 && in0 && y + k < y1) ? __ldg(row - 1) : 0.0;
        rx[k] = (in1 && y + k < y1 && (lane == 31 || x + 2 >= lp.end[0])) ? __ldg(row + 2) : 0.0;
      }
#pragma unroll
      for (int k = 0; k < B; k++) {
        if (y + k >= y1) break;
        const double lft = __shfl_up_sync(0xffffffffu, c.y, 1);
        const double rgt = __shfl_down_sync(0xffffffffu, c.x, 1);
        const double l0 = lane == 0 ? lx[k] : lft;                                // A(x-1, y)
        const double r1 = (lane == 31 || x + 2 >= lp.end[0]) ? rx[k] : rgt;       // A(x+2, y)
        double *o = An + x + (long long)(y + k) * pn;
        if (in0) {
          const double v0 = 0.25f * (c.y + l0 + dn.x + up[k].x);  // A(1,0) + A(-1,0) + A(0,-1) + A(0,1) at x
          o[0] = v0;
          err = fmax(err, fabs(v0 - c.x));
        }
        if (in1) {
          const double v1 = 0.25f * (r1 + c.x + dn.y + up[k].y);  // the same at x + 1
          o[1] = v1;
          err = fmax(err, fabs(v1 - c.y));
        }
        dn = c;
        c = up[k];
      }
    }
  }
  __shared__ double smem[32];
  __shared__ int last;
  const int nblocks = gridDim.x * gridDim.y;
  const double b = block_reduce<double>(err, ACC_MAX, smem);
  const int bid = blockIdx.x + blockIdx.y * gridDim.x;
  if (threadIdx.x == 0) {
    reinterpret_cast<double *>(lp.red_scratch)[((size_t)vr.red_index * nblocks + bid) * OPSB_MAX_RED_DIM] = b;
    __threadfence();
    last = (atomicAdd(lp.red_counter, 1u) == (unsigned int)(nblocks - 1));
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  finish_grid_reduction<double>(vr, lp, nblocks, smem);
  if (threadIdx.x == 0) *lp.red_counter = 0u;
}

template <int X, int R, int B>
void launch_march2(const LoopParams &lp, cudaStream_t s) {
  const int nx = lp.end[0] - lp.start[0], ny = lp.end[1] - lp.start[1];
  const dim3 g((unsigned)std::max(1, (nx + 2 * X - 1) / (2 * X)), (unsigned)std::max(1, (ny + R - 1) / R));
  if ((long long)g.x * g.y > Runtime::kMaxRedBlocks)
    throw Error(E_UNSUPPORTED, "laplace2d/apply_stencil: range too large for one reduction");
  apply_stencil_march2<X, R, B><<<g, X, 0, s>>>(lp);
}

template <int X, int R, int B>
void launch_march(const LoopParams &lp, cudaStream_t s) {
  const int nx = lp.end[0] - lp.start[0], ny = lp.end[1] - lp.start[1];
  const dim3 g((unsigned)std::max(1, (nx + X - 1) / X), (unsigned)std::max(1, (ny + R - 1) / R));
  if ((long long)g.x * g.y > Runtime::kMaxRedBlocks)
    throw Error(E_UNSUPPORTED, "laplace2d/apply_stencil: range too large for one reduction");
  apply_stencil_march<X, R, B><<<g, X, 0, s>>>(lp);
}

struct apply_stencil {
  static constexpr const char *kname = "laplace2d/apply_stencil";
  __device__ void operator()(const ACC2<double> &A, ACC2<double> &Anew, RED<double> &error) const {
    Anew(0, 0) = 0.25f * (A(1, 0) + A(-1, 0) + A(0, -1) + A(0, 1));
    *error = fmax(*error, fabs(Anew(0, 0) - A(0, 0)));
  }
  // The column march needs A read through the plain 5-point stencil (the
  // only stencil this kernel is used with); its strides come from the
  // argument views, so any range and pitch work.
  static void launch(const LoopParams &lp, dim3 g_hint, dim3 b_hint, cudaStream_t s) {
    const ArgView &va = lp.a[0], &vn = lp.a[1];
    if (va.sx != 1 || va.sy != va.ay || va.mg || vn.sx != 1 || vn.sy != vn.ay || vn.mg || lp.ndim != 2) {
      exec_loop<apply_stencil><<<g_hint, b_hint, 0, s>>>(lp);  // strided or multigrid stencils: the generic path
      return;
    }
    // pairs of columns need 16-byte aligned loads: an even start column, an
    // even pitch and an aligned dat origin; otherwise one column per thread
    const bool pairs = (lp.start[0] % 2) == 0 && (va.ay % 2) == 0 &&
                       (reinterpret_cast<uintptr_t>(va.ptr) % 16) == 0;
    if (pairs)
      launch_march2<256, 32, 4>(lp, s);  // 4.83 TB/s at 4096^2 (generic executor 3.93)
    else
      launch_march<256, 32, 4>(lp, s);   // 4.20 TB/s
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
