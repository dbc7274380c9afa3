// Allocation-free Laplace sweep.
//
// Some callers cannot allocate device memory at the point where they need a
// sweep: code running inside a memory pool or arena that another framework
// owns (cudaMalloc would fragment it or bypass its accounting), code between
// a stream-capture begin/end that must not add allocation nodes, and
// latency-critical loops where an allocator call (and the implicit
// synchronisation cudaFree carries) is unacceptable. For them this file
// provides one Jacobi sweep of the Laplace stencil with its max|delta|
// reduction, the same arithmetic as loop kernel "laplace2d/apply_stencil",
// whose only scratch memory (per-block partial maxima and a blocks-done
// counter) is a fixed file-scope __device__ array.
//
// Limits and rules (also stated in include/ops_b200.h):
//   * at most kMaxBlocks blocks share the scratch, which bounds the grid;
//     imax and jmax must be <= kMaxExtent, larger sizes are rejected;
//   * the scratch lives in every GPU that loads this library, for the life
//     of the process (kMaxBlocks doubles plus one counter, about 32 KiB);
//   * every call shares that one array: calls that may overlap on the GPU
//     (different streams, or different host threads on one device) race and
//     must be serialised by the caller;
//   * the first call on each device resolves the array's device address with
//     cudaGetSymbolAddress while that device is current; make that first
//     call before any stream capture that should contain a sweep.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/ops_b200.h"

namespace {

constexpr int kMaxBlocks = 4096;
constexpr int kMaxExtent = 65536;
constexpr int kMaxDevices = 64;
constexpr int kBX = 128, kBY = 2;

// Scratch: [0, kMaxBlocks) block partials, then the blocks-done counter.
static __device__ __align__(256) double g_noalloc_scratch[kMaxBlocks + 1];

// Device addresses of the scratch, one per device (host code cannot use the
// symbol itself: on the host it names a shadow, not device memory). Read
// without the lock on every call, so each slot is atomic: the first call on
// a device publishes the address with release order after looking it up,
// later calls (any thread) read it with acquire order.
std::atomic<double *> g_scratch_ptr[kMaxDevices];
std::mutex g_setup_mutex;
thread_local char g_err[256] = "no error";

__global__ void __launch_bounds__(kBX *kBY)
    laplace_sweep_noalloc_kernel(const double *__restrict__ A, double *__restrict__ Anew, long long pitch, int imax,
                                 int jmax, double *scratch, double *max_delta) {
  const int x = blockIdx.x * kBX + threadIdx.x;
  double err = -1.7976931348623157e308;
  if (x < imax) {
    for (int y = blockIdx.y * kBY + threadIdx.y; y < jmax; y += gridDim.y * kBY) {
      const double *a = A + x + (long long)y * pitch;
      // Same expression and order as apps/c/laplace2d_tutorial/step7/laplace_kernels.h:22-26.
      const double v = 0.25f * (a[1] + a[-1] + a[-pitch] + a[pitch]);
      Anew[x + (long long)y * pitch] = v;
      err = fmax(err, fabs(v - a[0]));
    }
  }
  // Block maximum: warp shuffles, then one value per warp in shared memory.
  for (int o = 16; o > 0; o >>= 1) err = fmax(err, __shfl_down_sync(0xffffffffu, err, o));
  __shared__ double warp_max[kBX * kBY / 32];
  __shared__ int last;
  const int tid = threadIdx.x + threadIdx.y * kBX;
  if ((tid & 31) == 0) warp_max[tid >> 5] = err;
  __syncthreads();
  const int nblocks = gridDim.x * gridDim.y;
  unsigned int *counter = reinterpret_cast<unsigned int *>(scratch + kMaxBlocks);
  if (tid == 0) {
    double m = warp_max[0];
    for (int w = 1; w < kBX * kBY / 32; w++) m = fmax(m, warp_max[w]);
    scratch[blockIdx.x + blockIdx.y * gridDim.x] = m;
    __threadfence();
    last = (atomicAdd(counter, 1u) == (unsigned int)(nblocks - 1));
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // The last block folds the partials in a fixed order and re-arms the counter.
  double m = -1.7976931348623157e308;
  for (int b = tid; b < nblocks; b += kBX * kBY) m = fmax(m, scratch[b]);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((tid & 31) == 0) warp_max[tid >> 5] = m;
  __syncthreads();
  if (tid == 0) {
    double r = warp_max[0];
    for (int w = 1; w < kBX * kBY / 32; w++) r = fmax(r, warp_max[w]);
    *max_delta = r;
    *counter = 0u;
  }
}

int fail(int code, const char *msg) {
  snprintf(g_err, sizeof(g_err), "%s", msg);
  return code;
}

}  // namespace

extern "C" const char *ops_b200_noalloc_last_error(void) { return g_err; }

extern "C" int ops_b200_laplace_sweep_noalloc(int imax, int jmax, const double *A, double *Anew, long long pitch,
                                              double *max_delta, void *stream) {
  if (imax <= 0 || jmax <= 0 || !A || !Anew || !max_delta)
    return fail(OPS_B200_ERR_ARG, "laplace_sweep_noalloc: imax, jmax must be positive and pointers non-NULL");
  if (imax > kMaxExtent || jmax > kMaxExtent)
    return fail(OPS_B200_ERR_ARG, "laplace_sweep_noalloc: imax and jmax must be <= 65536 (fixed scratch size)");
  if (pitch < (long long)imax + 2)
    return fail(OPS_B200_ERR_ARG, "laplace_sweep_noalloc: pitch must be at least imax + 2");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(OPS_B200_ERR_CUDA, "laplace_sweep_noalloc: no current CUDA device");
  double *scratch = g_scratch_ptr[dev].load(std::memory_order_acquire);
  if (!scratch) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    scratch = g_scratch_ptr[dev].load(std::memory_order_relaxed);
    if (!scratch) {
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return fail(OPS_B200_ERR_CUDA, "laplace_sweep_noalloc: cudaGetSymbolAddress failed for the scratch array");
      scratch = static_cast<double *>(p);
      g_scratch_ptr[dev].store(scratch, std::memory_order_release);
    }
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The counter must start at zero; a previous call re-arms it, this makes
  // a call that followed an aborted one safe too.
  if (cudaMemsetAsync(scratch + kMaxBlocks, 0, sizeof(double), s) != cudaSuccess)
    return fail(OPS_B200_ERR_CUDA, "laplace_sweep_noalloc: clearing the counter failed");
  const int gx = (imax + kBX - 1) / kBX;
  int gy = (jmax + kBY - 1) / kBY;
  const int cap = kMaxBlocks / gx;
  if (gy > cap) gy = cap;
  if (gy > 148 * 16 / gx + 1) gy = 148 * 16 / gx + 1;
  if (gy < 1) gy = 1;
  laplace_sweep_noalloc_kernel<<<dim3(gx, gy), dim3(kBX, kBY), 0, s>>>(A, Anew, pitch, imax, jmax, scratch,
                                                                        max_delta);
  if (cudaGetLastError() != cudaSuccess) return fail(OPS_B200_ERR_CUDA, "laplace_sweep_noalloc: launch failed");
  return OPS_B200_OK;
}
