// C-ABI of the learned-preconditioner building blocks (no reference
// counterpart: the reference has no learned preconditioner).
#include <cuda_runtime.h>

#include <functional>
#include <mutex>
#include <string>

#include "../../include/ops_b200.h"
#include "conv_tc.cuh"
#include "runtime.h"

namespace opsb {
int capi_guard(const std::function<int()> &f);

namespace cnn {
// One device error word per device for the convolution kernels' bounded waits.
int *error_word() {
  static std::mutex mu;
  static int *words[64] = {nullptr};
  int dev = 0;
  OPSB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw Error(E_CUDA, "device index out of range");
  std::lock_guard<std::mutex> lk(mu);
  if (!words[dev]) {
    OPSB_CUDA(cudaMalloc(&words[dev], 64));
    OPSB_CUDA(cudaMemset(words[dev], 0, 64));
  }
  return words[dev];
}
}  // namespace cnn
}  // namespace opsb

extern "C" int ops_b200_conv3x3_bf16(const void *x, const void *w, const float *bias, const void *mask, void *y,
                                     int n, int h, int wd, int cin, int cout, int mode, void *stream) {
  using namespace opsb;
  return capi_guard([&] {
    if (mode < 0 || mode > 3) throw Error(E_ARG, "conv mode must be 0..3");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int *err = cnn::error_word();
    OPSB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    cudaError_t e = cnn::conv3x3(reinterpret_cast<const __nv_bfloat16 *>(x), reinterpret_cast<const __nv_bfloat16 *>(w),
                                 n, h, wd, cin, cout, bias, reinterpret_cast<const __nv_bfloat16 *>(mask),
                                 reinterpret_cast<__nv_bfloat16 *>(y), mode, err, s);
    if (e == cudaErrorInvalidValue || e == cudaErrorMisalignedAddress)
      throw Error(E_ARG, std::string("conv3x3: unsupported shape or alignment: ") + cudaGetErrorString(e));
    OPSB_CUDA(e);
    int h_err = 0;
    OPSB_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    OPSB_CUDA(cudaStreamSynchronize(s));
    if (h_err) throw Error(E_TIMEOUT, "conv3x3: a pipeline wait expired (code " + std::to_string(h_err) + ")");
    return 0;
  });
}
