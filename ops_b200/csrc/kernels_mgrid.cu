// Multigrid test kernels (apps/c/mgrid/mgrid_kernels.h): populate a level
// with its index, restrict (fine -> coarse) and prolong (coarse -> fine) by
// plain injection through restrict/prolong stencils, and the app's own
// checks of the results. The restrict and prolong kernels state `mgrid` so
// their accessors map the point's index through the multigrid stencils.
// Loop names are "mgrid/<reference kernel name>".
#include "runtime.h"

namespace opsb {
namespace mgrid {

using D = ACC2<double>;

#define MG_LOOP(NAME) static constexpr const char *kname = "mgrid/" #NAME

struct mgrid_populate_kernel_1 {  // :5
  MG_LOOP(mgrid_populate_kernel_1);
  __device__ void operator()(D &val, const IDX &idx) const { val(0, 0) = (double)(idx[0] + 6 * idx[1]); }
};
struct mgrid_populate_kernel_2 {  // :9
  MG_LOOP(mgrid_populate_kernel_2);
  __device__ void operator()(D &val, const IDX &idx) const { val(0, 0) = (double)(idx[0] + 4 * idx[1]); }
};
struct mgrid_populate_kernel_3 {  // :13
  MG_LOOP(mgrid_populate_kernel_3);
  __device__ void operator()(D &val, const IDX &idx) const { val(0, 0) = (double)(idx[0] + 24 * idx[1]); }
};
struct mgrid_restrict_kernel {  // :17
  MG_LOOP(mgrid_restrict_kernel);
  static constexpr bool mgrid = true;
  __device__ void operator()(const D &fine, D &coarse, const IDX &) const { coarse(0, 0) = fine(0, 0); }
};
struct mgrid_prolong_kernel {  // :22
  MG_LOOP(mgrid_prolong_kernel);
  static constexpr bool mgrid = true;
  __device__ void operator()(const D &coarse, D &fine, const IDX &) const { fine(0, 0) = coarse(0, 0); }
};
// The checks: a level prolonged twice by 2 from the 6-wide coarse level
// holds x/4 + (y/4) * (sizex/4), with periodic neighbours (:27-56); a level
// restricted twice by 2 from the 24-wide fine one holds 4x + 4y * sizex
// (:58-66). Each point overwrites its thread's flag, the flags combine by
// max.
struct prolong_check {
  MG_LOOP(prolong_check);
  __device__ void operator()(const D &val, const IDX &idx, RED<int> &err, const int *sizex, const int *sizey) const {
    int lerr = 0;
    lerr |= (val(0, 0) != idx[0] / 4 + (idx[1] / 4) * (*sizex / 4));
    int xm = (idx[0] - 1) < 0 ? *sizex - 1 : idx[0] - 1;
    int xp = (idx[0] + 1) >= *sizex ? 0 : idx[0] + 1;
    int ym = (idx[1] - 1) < 0 ? *sizey - 1 : idx[1] - 1;
    int yp = (idx[1] + 1) >= *sizey ? 0 : idx[1] + 1;
    lerr |= (val(1, 0) != xp / 4 + (idx[1] / 4) * (*sizex / 4));
    lerr |= (val(-1, 0) != xm / 4 + (idx[1] / 4) * (*sizex / 4));
    lerr |= (val(0, 1) != idx[0] / 4 + (yp / 4) * (*sizex / 4));
    lerr |= (val(0, -1) != idx[0] / 4 + (ym / 4) * (*sizex / 4));
    *err = lerr != 0 ? 1 : 0;
  }
};
struct restrict_check {
  MG_LOOP(restrict_check);
  __device__ void operator()(const D &val, const IDX &idx, RED<int> &err, const int *sizex) const {
    *err = (val(0, 0) != idx[0] * 4 + idx[1] * 4 * *sizex) ? 1 : 0;
  }
};

#define REG(K) OPSB_REGISTER_LOOP(K);
REG(mgrid_populate_kernel_1) REG(mgrid_populate_kernel_2) REG(mgrid_populate_kernel_3) REG(mgrid_restrict_kernel)
REG(mgrid_prolong_kernel) REG(prolong_check) REG(restrict_check)

}  // namespace mgrid
}  // namespace opsb
