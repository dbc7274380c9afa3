// Learned multigrid preconditioner for the TeaLeaf heat operator (no
// reference counterpart): a 4-level U-Net-shaped CNN that maps a residual r
// and the operator's face coefficients to an approximation of the error
// e = A^-1 r, trained on residual/error pairs from Jacobi-PCG and applied
// inside flexible CG.
//
// Network (NHWC BF16 activations, FP32 accumulation, 3x3 convs on tcgen05):
//   x0  = features(r, Kx, Ky)                       16 ch (5 used), H x W
//   e0  = relu(C0 x0)                               16 ch
//   e1  = relu(C1b relu(C1a pool e0))               32 ch, H/2
//   e2  = relu(C2b relu(C2a pool e1))               64 ch, H/4
//   h3  = relu(C3b relu(C3a pool e2))               64 ch, H/8
//   h2  = relu(C2u (up h3 + e2))                    32 ch, H/4
//   h1  = relu(C1u (up h2 + e1))                    16 ch, H/2
//   h0  = relu(C0u (up h1 + e0))                    16 ch, H
//   y   = wout . h0 + bout                          1 ch, FP32
//   M(r) = z + s y,  z = r / diag(A),  s = rms(r) per image
// Features: r / s and the four normalised face weights a/D, b/D, c/D, d/D
// (a = rx Kx(i), b = rx Kx(i+1), c = ry Ky(j), d = ry Ky(j+1),
// D = 1 + a + b + c + d = diag(A)). The output layer starts at zero, so an
// untrained network is the Jacobi preconditioner.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <vector>

namespace opsb {
namespace lmg {

// A batch of FP64 fields sharing one layout: element (n, y, x) of the
// interior is at ptr[n * image + y * pitch + x]; Kx and Ky reach x = W and
// y = H (the east and north faces of the last cells).
struct Fields {
  int n = 0, h = 0, w = 0;
  long long pitch = 0, image = 0;
  const double *r = nullptr, *Kx = nullptr, *Ky = nullptr;
  double rx = 0, ry = 0;
};

constexpr int kLayers = 10;
enum { LOSS_L2 = 0, LOSS_ANORM = 1 };

class Net {
 public:
  explicit Net(unsigned long long seed);
  ~Net();
  Net(const Net &) = delete;
  Net &operator=(const Net &) = delete;

  static int num_params();
  // FP32 parameters: per conv layer W [9][cout][cin] then b [cout]; then
  // wout [16], bout.
  void get_params(float *host) const;
  void set_params(const float *host);
  void get_grads(float *host) const;

  // z = M(r) written to out (FP64, same layout as f). Allocates activation
  // buffers for (n, h, w) on first use.
  void apply(const Fields &f, double *out, cudaStream_t s);
  // Forward + backward for a batch with targets e (same layout as f);
  // gradients of loss = mean_n ||M(r_n) - e_n||^2 / ||e_n||^2 (LOSS_L2) or of
  // the same ratio in the A-norm, (d.Ad) / (e.Ae) with d = M(r_n) - e_n
  // (LOSS_ANORM), land in the gradient buffer. Returns the loss.
  double loss_and_grad(const Fields &f, const double *e, int kind, cudaStream_t s);
  // One Adam step on the stored gradients.
  void adam(double lr, cudaStream_t s);
  long long launches() const { return launches_; }

  struct Impl;

 private:
  Impl *m_;
  long long launches_ = 0;
};

}  // namespace lmg
}  // namespace opsb
