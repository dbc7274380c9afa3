// Laplace Jacobi driver: the loop sequence of
// apps/c/laplace2d_tutorial/step7/laplace2d.cpp:41-124 on the OPS-B200
// runtime, with the boundary ring supplied by the caller.
#include <cstring>
#include <functional>

#include "../../include/ops_b200.h"
#include "runtime.h"

namespace opsb {
int capi_guard(const std::function<int()> &f);
namespace laplace {
struct apply_stencil;
struct copy;
}  // namespace laplace

// Declared in kernels_laplace.cu.
void laplace_par_loop_apply(int block, const int *range, int dA, int dAnew, int s5, int s0, int h_err);
void laplace_par_loop_copy(int block, const int *range, int dA, int dAnew, int s0);

}  // namespace opsb

extern "C" int ops_b200_app_laplace2d(int imax, int jmax, int warmup, int iters, const double *field_in,
                                      double *field_out, double *err_per_iter, double *device_seconds) {
  using namespace opsb;
  return capi_guard([&] {
    if (imax <= 0 || jmax <= 0 || iters < 0 || warmup < 0 || !field_in) throw Error(E_ARG, "bad Laplace arguments");
    Runtime &r = Runtime::get();
    if (!r.initialized()) r.init(0, 0);
    ReleaseScope scope(r);
    int block = r.decl_block(2, "my_grid");
    int size[] = {imax, jmax}, base[] = {0, 0}, d_m[] = {-1, -1}, d_p[] = {1, 1};
    int dA = r.decl_dat(block, 1, size, base, d_m, d_p, field_in, 8, "double", "A");
    int dAnew = r.decl_dat(block, 1, size, base, d_m, d_p, field_in, 8, "double", "Anew");
    int s00[] = {0, 0};
    int s0 = r.decl_stencil(2, 1, s00, nullptr, "0,0");
    int s5pt[] = {0, 0, 1, 0, -1, 0, 0, 1, 0, -1};
    int s5 = r.decl_stencil(2, 5, s5pt, nullptr, "5pt");
    int h_err = r.decl_reduction(sizeof(double), "double", "error");
    r.partition("");  // laplace2d.cpp:61
    r.decl_const("imax", 1, "int", &imax);
    r.decl_const("jmax", 1, "int", &jmax);

    EventPair ev;
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    int interior[] = {0, imax, 0, jmax};
    double error = 1.0;
    for (int it = 0; it < warmup + iters; it++) {
      if (it == warmup) {
        r.execute();
        OPSB_CUDA(cudaEventRecord(e0, r.stream()));
      }
      laplace_par_loop_apply(block, interior, dA, dAnew, s5, s0, h_err);
      r.reduction_result(h_err, &error);
      if (err_per_iter) err_per_iter[it] = error;
      laplace_par_loop_copy(block, interior, dA, dAnew, s0);
    }
    if (warmup + iters == 0 || iters == 0) OPSB_CUDA(cudaEventRecord(e0, r.stream()));
    r.execute();
    OPSB_CUDA(cudaEventRecord(e1, r.stream()));
    OPSB_CUDA(cudaEventSynchronize(e1));
    if (device_seconds) *device_seconds = ev.ms() * 1e-3;
    if (field_out) {
      // partitioned across ranks: this rank's owned rows, in place in the
      // whole (imax + 2) x (jmax + 2) array
      int disp[2], ext[2];
      r.dat_get_extents(dA, disp, ext);
      r.dat_fetch_data(dA, field_out + (size_t)disp[1] * (imax + 2), r.dat_data_bytes(dA));
    }
    scope.release();
    return 0;
  });
}
