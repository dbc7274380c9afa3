// 3x3 convolution (stride 1, zero padding 1) as an implicit GEMM on the
// 5th-generation tensor cores (tcgen05.mma kind::f16, BF16 operands, FP32
// accumulators in tensor memory), for the learned multigrid preconditioner.
//
// Layouts: activations NHWC BF16 [N][H][W][C]; weights [9][Cout][Cin] BF16
// with tap = (dy + 1) * 3 + (dx + 1); bias FP32 [Cout].
//
// GEMM view per tile: M = 128 output pixels (a TW x TH patch, TW * TH = 128),
// N = Cout, K = 9 * Cin. For each tap the A operand is the input patch shifted
// by (dx, dy): one TMA tiled load of a (Cin, TW, TH, 1) box whose start may lie
// outside the image, so the padding comes from the TMA zero fill. Each pixel
// row of the box is Cin * 2 bytes, loaded with the swizzle of that width
// (32, 64 or 128 bytes), which is the K-major canonical layout the MMA
// descriptor names; K steps of 16 inside a row advance the descriptor start
// address by 32 bytes. All nine weight tiles stay resident in shared memory.
//
// Warp roles (192 threads): warp 0 issues the TMA loads (and owns the tensor
// memory allocation), warp 1 issues the MMAs from one thread, warps 2-5 drain
// the accumulators (each warp reads its 32-lane quarter of tensor memory),
// add the bias, apply ReLU or a gradient mask and store BF16. Four accumulator
// buffers let the epilogues of earlier tiles overlap the MMAs of later ones,
// and several CTAs share an SM where shared and tensor memory allow. Every
// mbarrier wait is bounded: on expiry the kernel records an error code,
// stops issuing work, waits (bounded) for its own copies in flight, frees its
// tensor memory and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace opsb {
namespace cnn {

enum ConvMode {
  CONV_BIAS_RELU = 0,   // y = relu(conv(x) + b)
  CONV_BIAS = 1,        // y = conv(x) + b
  CONV_MASK = 2,        // y = conv(x) * (m > 0), m a BF16 tensor shaped like y (ReLU backward)
  CONV_PLAIN = 3        // y = conv(x)
};

struct ConvArgs {
  int n, h, w;          // images, rows, columns
  int tw, th;           // pixel patch per tile (tw * th == 128)
  int tiles_x, tiles_y, tiles;
  const float *bias;    // [Cout] (modes 0, 1)
  const __nv_bfloat16 *mask;  // [N][H][W][Cout] (mode 2)
  __nv_bfloat16 *y;     // [N][H][W][Cout]
  int mode;
  int *err;             // device error word (0 = fine)
};

// Launches y = conv3x3(x, w) (+ epilogue) on stream s. x, w, y are device
// pointers; the tensor maps are encoded on the host per call. Returns
// cudaErrorInvalidValue for unsupported shapes, cudaErrorMisalignedAddress
// for pointers not 16-byte aligned, else the launch status.
cudaError_t conv3x3(const __nv_bfloat16 *x, const __nv_bfloat16 *w, int n, int h, int wd, int cin, int cout,
                    const float *bias, const __nv_bfloat16 *mask, __nv_bfloat16 *y, int mode, int *err,
                    cudaStream_t s);

}  // namespace cnn
}  // namespace opsb
