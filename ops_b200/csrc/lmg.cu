// Learned multigrid preconditioner: network, training step and application
// (see lmg.h for the architecture). The 3x3 convolutions, forward and
// input-gradient, run on the tcgen05 kernel of conv_tc.cu; the input gradient
// of a convolution is the convolution of the output gradient with the
// weights flipped in space and transposed in channels. Everything else is
// bandwidth-bound elementwise work on CUDA cores, NHWC with 8 channels
// (16 bytes) per thread. Weight gradients are per-CTA partial sums added in
// a fixed order, so a training step is reproducible run to run.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "conv_tc.cuh"
#include "lmg.h"
#include "runtime.h"

namespace opsb {
namespace cnn {
int *error_word();
}
namespace lmg {
namespace {

struct LayerDef {
  int cin, cout;
};
constexpr LayerDef kDefs[kLayers] = {{16, 16}, {16, 32}, {32, 32}, {32, 64}, {64, 64},
                                     {64, 64}, {64, 64}, {64, 32}, {32, 16}, {16, 16}};
enum { C0 = 0, C1A, C1B, C2A, C2B, C3A, C3B, C2U, C1U, C0U };
constexpr int kFeat = 16;   // input channels (5 used)
constexpr int kT = 256;     // threads of the elementwise kernels
constexpr int kWgX = 128;   // pixel groups of the weight-gradient kernel
constexpr int kWgTile = 128;  // pixels per weight-gradient tile (16 x 8)

using bf16 = __nv_bfloat16;

struct Offsets {
  int w[kLayers], b[kLayers], wout, bout, total;
  Offsets() {
    int o = 0;
    for (int l = 0; l < kLayers; l++) {
      w[l] = o;
      o += 9 * kDefs[l].cin * kDefs[l].cout;
      b[l] = o;
      o += kDefs[l].cout;
    }
    wout = o;
    o += 16;
    bout = o;
    o += 1;
    total = o;
  }
};
const Offsets &offs() {
  static Offsets o;
  return o;
}

__device__ __forceinline__ void ld8(const bf16 *p, float *v) {
  uint4 u = *reinterpret_cast<const uint4 *>(p);
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    float2 f = __bfloat1622float2(h[k]);
    v[2 * k] = f.x;
    v[2 * k + 1] = f.y;
  }
}
__device__ __forceinline__ void st8(bf16 *p, const float *v) {
  uint4 u;
  __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
  for (int k = 0; k < 4; k++) h[k] = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
  *reinterpret_cast<uint4 *>(p) = u;
}

__device__ __forceinline__ double block_sum_d(double v, double *sm) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sm[wid] = v;
  __syncthreads();
  v = 0.0;
  if (wid == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sm[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// Face weights and diagonal of A at interior cell (x, y) of image n.
struct Coef {
  double a, b, c, d, D;
};
__device__ __forceinline__ Coef coef(const Fields &f, int n, int y, int x) {
  const long long i = n * f.image + (long long)y * f.pitch + x;
  Coef k;
  k.a = f.rx * f.Kx[i];
  k.b = f.rx * f.Kx[i + 1];
  k.c = f.ry * f.Ky[i];
  k.d = f.ry * f.Ky[i + f.pitch];
  k.D = 1.0 + k.a + k.b + k.c + k.d;
  return k;
}

// Per image, per block: partial sums of r^2.
__global__ void k_zsq(Fields f, double *part) {
  __shared__ double sm[kT / 32];
  const int n = blockIdx.y;
  const int hw = f.h * f.w;
  double acc = 0.0;
  for (int p = blockIdx.x * kT + threadIdx.x; p < hw; p += gridDim.x * kT) {
    const int y = p / f.w, x = p - y * f.w;
    const double r = f.r[n * f.image + (long long)y * f.pitch + x];
    acc += r * r;
  }
  acc = block_sum_d(acc, sm);
  if (threadIdx.x == 0) part[n * gridDim.x + blockIdx.x] = acc;
}

// s[n] = rms(r) (1 when the residual is zero), partials added in block order.
__global__ void k_scale(const double *part, int nblk, int hw, double *s, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double t = 0.0;
  for (int b = 0; b < nblk; b++) t += part[i * nblk + b];
  const double v = sqrt(t / (double)hw);
  s[i] = v > 0.0 ? v : 1.0;
}

__global__ void k_features(Fields f, const double *s, bf16 *x0) {
  const long long total = (long long)f.n * f.h * f.w;
  for (long long p = (long long)blockIdx.x * kT + threadIdx.x; p < total; p += (long long)gridDim.x * kT) {
    const int n = (int)(p / ((long long)f.h * f.w));
    const int rem = (int)(p - (long long)n * f.h * f.w);
    const int y = rem / f.w, x = rem - y * f.w;
    const Coef k = coef(f, n, y, x);
    float v[16] = {0};
    v[0] = (float)(f.r[n * f.image + (long long)y * f.pitch + x] / s[n]);
    v[1] = (float)(k.a / k.D);
    v[2] = (float)(k.b / k.D);
    v[3] = (float)(k.c / k.D);
    v[4] = (float)(k.d / k.D);
    st8(x0 + p * kFeat, v);
    st8(x0 + p * kFeat + 8, v + 8);
  }
}

// 2x2 average pooling, C channels.
__global__ void k_pool(const bf16 *in, bf16 *out, int n, int h, int w, int C) {
  const int h2 = h / 2, w2 = w / 2, g = C / 8;
  const long long total = (long long)n * h2 * w2 * g;
  for (long long t = (long long)blockIdx.x * kT + threadIdx.x; t < total; t += (long long)gridDim.x * kT) {
    const int cg = (int)(t % g);
    long long p = t / g;
    const int X = (int)(p % w2);
    p /= w2;
    const int Y = (int)(p % h2);
    const int img = (int)(p / h2);
    float acc[8] = {0}, v[8];
    for (int dy = 0; dy < 2; dy++)
      for (int dx = 0; dx < 2; dx++) {
        ld8(in + (((long long)img * h + 2 * Y + dy) * w + 2 * X + dx) * C + cg * 8, v);
#pragma unroll
        for (int k = 0; k < 8; k++) acc[k] += v[k];
      }
#pragma unroll
    for (int k = 0; k < 8; k++) acc[k] *= 0.25f;
    st8(out + (((long long)img * h2 + Y) * w2 + X) * C + cg * 8, acc);
  }
}

// out = up2(coarse) + skip, fine grid n x h x w, C channels.
__global__ void k_up_add(const bf16 *coarse, const bf16 *skip, bf16 *out, int n, int h, int w, int C) {
  const int g = C / 8;
  const long long total = (long long)n * h * w * g;
  for (long long t = (long long)blockIdx.x * kT + threadIdx.x; t < total; t += (long long)gridDim.x * kT) {
    const int cg = (int)(t % g);
    long long p = t / g;
    const int x = (int)(p % w);
    p /= w;
    const int y = (int)(p % h);
    const int img = (int)(p / h);
    float a[8], b[8];
    ld8(coarse + (((long long)img * (h / 2) + y / 2) * (w / 2) + x / 2) * C + cg * 8, a);
    const long long fi = (((long long)img * h + y) * w + x) * C + cg * 8;
    ld8(skip + fi, b);
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] += b[k];
    st8(out + fi, a);
  }
}

// Gradient through up2: coarse (n, h/2, w/2) = sum of its four children,
// times (mask > 0) (the ReLU of the layer that produced the coarse tensor).
__global__ void k_upT_mask(const bf16 *fine, const bf16 *mask, bf16 *out, int n, int h, int w, int C) {
  const int h2 = h / 2, w2 = w / 2, g = C / 8;
  const long long total = (long long)n * h2 * w2 * g;
  for (long long t = (long long)blockIdx.x * kT + threadIdx.x; t < total; t += (long long)gridDim.x * kT) {
    const int cg = (int)(t % g);
    long long p = t / g;
    const int X = (int)(p % w2);
    p /= w2;
    const int Y = (int)(p % h2);
    const int img = (int)(p / h2);
    float acc[8] = {0}, v[8], m[8];
    for (int dy = 0; dy < 2; dy++)
      for (int dx = 0; dx < 2; dx++) {
        ld8(fine + (((long long)img * h + 2 * Y + dy) * w + 2 * X + dx) * C + cg * 8, v);
#pragma unroll
        for (int k = 0; k < 8; k++) acc[k] += v[k];
      }
    const long long ci = (((long long)img * h2 + Y) * w2 + X) * C + cg * 8;
    ld8(mask + ci, m);
#pragma unroll
    for (int k = 0; k < 8; k++) acc[k] = m[k] > 0.0f ? acc[k] : 0.0f;
    st8(out + ci, acc);
  }
}

// out = (a + 0.25 * up2(b)) * (mask > 0): the gradient reaching a tensor that
// feeds both a skip connection (a) and a 2x2 average pool (b, coarse).
__global__ void k_add_poolT_mask(const bf16 *a, const bf16 *b, const bf16 *mask, bf16 *out, int n, int h, int w,
                                 int C) {
  const int g = C / 8;
  const long long total = (long long)n * h * w * g;
  for (long long t = (long long)blockIdx.x * kT + threadIdx.x; t < total; t += (long long)gridDim.x * kT) {
    const int cg = (int)(t % g);
    long long p = t / g;
    const int x = (int)(p % w);
    p /= w;
    const int y = (int)(p % h);
    const int img = (int)(p / h);
    const long long fi = (((long long)img * h + y) * w + x) * C + cg * 8;
    float va[8], vb[8], m[8];
    ld8(a + fi, va);
    ld8(b + (((long long)img * (h / 2) + y / 2) * (w / 2) + x / 2) * C + cg * 8, vb);
    ld8(mask + fi, m);
#pragma unroll
    for (int k = 0; k < 8; k++) va[k] = m[k] > 0.0f ? va[k] + 0.25f * vb[k] : 0.0f;
    st8(out + fi, va);
  }
}

// Output layer: y = wout . h0 + bout; M(r) = z + s y. Writes M(r) to `out`
// (FP64, field layout) and/or the prediction to `pred` (FP32, dense n*h*w).
__global__ void k_out(Fields f, const double *s, const bf16 *h0, const float *params, int wout_off,
                      double *out, long long out_image, long long out_pitch, float *pred) {
  __shared__ float wsm[17];
  if (threadIdx.x < 17) wsm[threadIdx.x] = params[wout_off + threadIdx.x];
  __syncthreads();
  const long long total = (long long)f.n * f.h * f.w;
  for (long long p = (long long)blockIdx.x * kT + threadIdx.x; p < total; p += (long long)gridDim.x * kT) {
    const int n = (int)(p / ((long long)f.h * f.w));
    const int rem = (int)(p - (long long)n * f.h * f.w);
    const int y = rem / f.w, x = rem - y * f.w;
    float v[16];
    ld8(h0 + p * 16, v);
    ld8(h0 + p * 16 + 8, v + 8);
    float acc = wsm[16];
#pragma unroll
    for (int c = 0; c < 16; c++) acc += wsm[c] * v[c];
    const Coef k = coef(f, n, y, x);
    const double z = f.r[n * f.image + (long long)y * f.pitch + x] / k.D;
    const double m = z + s[n] * (double)acc;
    if (out) out[n * out_image + (long long)y * out_pitch + x] = m;
    if (pred) pred[p] = (float)m;
  }
}

// d = pred - e in place (FP32, dense n x h x w); per-image partials of d.d
// and e.e (the L2 loss).
__global__ void k_diff(Fields f, float *pd, const double *e, double *part) {
  __shared__ double sm[kT / 32];
  const int n = blockIdx.y, hw = f.h * f.w;
  double a = 0.0, b = 0.0;
  for (int p = blockIdx.x * kT + threadIdx.x; p < hw; p += gridDim.x * kT) {
    const int y = p / f.w, x = p - y * f.w;
    const double ev = e[n * f.image + (long long)y * f.pitch + x];
    const double d = (double)pd[(long long)n * hw + p] - ev;
    pd[(long long)n * hw + p] = (float)d;
    a += d * d;
    b += ev * ev;
  }
  a = block_sum_d(a, sm);
  b = block_sum_d(b, sm);
  if (threadIdx.x == 0) {
    part[(n * gridDim.x + blockIdx.x) * 2] = a;
    part[(n * gridDim.x + blockIdx.x) * 2 + 1] = b;
  }
}

// A-norm loss: G = A d (the heat operator on the interior, d zero outside)
// and per-image partials of d.(A d) and e.(A e).
__global__ void k_anorm(Fields f, const float *d, const double *e, float *G, double *part) {
  __shared__ double sm[kT / 32];
  const int n = blockIdx.y, hw = f.h * f.w;
  const float *dn = d + (long long)n * hw;
  double a = 0.0, b = 0.0;
  for (int p = blockIdx.x * kT + threadIdx.x; p < hw; p += gridDim.x * kT) {
    const int y = p / f.w, x = p - y * f.w;
    const Coef k = coef(f, n, y, x);
    const double dc = dn[p];
    const double dw = x > 0 ? dn[p - 1] : 0.0, de = x + 1 < f.w ? dn[p + 1] : 0.0;
    const double ds = y > 0 ? dn[p - f.w] : 0.0, dnn = y + 1 < f.h ? dn[p + f.w] : 0.0;
    const double Ad = k.D * dc - k.a * dw - k.b * de - k.c * ds - k.d * dnn;
    const long long i = n * f.image + (long long)y * f.pitch + x;
    const double Ae = k.D * e[i] - k.a * e[i - 1] - k.b * e[i + 1] - k.c * e[i - f.pitch] - k.d * e[i + f.pitch];
    G[(long long)n * hw + p] = (float)Ad;
    a += dc * Ad;
    b += e[i] * Ae;
  }
  a = block_sum_d(a, sm);
  b = block_sum_d(b, sm);
  if (threadIdx.x == 0) {
    part[(n * gridDim.x + blockIdx.x) * 2] = a;
    part[(n * gridDim.x + blockIdx.x) * 2 + 1] = b;
  }
}

// Per image: E[n] = ||e||^2 (or e.Ae); loss = mean_n d.d / E[n] (or d.Ad / E[n]) (one thread).
__global__ void k_loss_finish(const double *part, int nblk, int n, double *E, double *loss) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double L = 0.0;
  for (int i = 0; i < n; i++) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < nblk; k++) {
      a += part[(i * nblk + k) * 2];
      b += part[(i * nblk + k) * 2 + 1];
    }
    if (!(b > 0.0)) b = 1.0;
    E[i] = b;
    L += a / b;
  }
  *loss = L / (double)n;
}

// dL/dy = (2 / n) s G / E with G = pred - e (L2) or A (pred - e) (A-norm),
// then through the output layer: g0u = dy * wout * (h0 > 0); per-block
// partials of dwout = sum dy h0, dbout = sum dy.
__global__ void k_out_bwd(Fields f, const double *s, const double *E, const float *G, const bf16 *h0,
                          const float *params, int wout_off, bf16 *g0u, float *part) {
  __shared__ float wsm[16];
  __shared__ double sm[kT / 32];
  if (threadIdx.x < 16) wsm[threadIdx.x] = params[wout_off + threadIdx.x];
  __syncthreads();
  double acc[17];
#pragma unroll
  for (int c = 0; c < 17; c++) acc[c] = 0.0;
  const long long total = (long long)f.n * f.h * f.w;
  for (long long p = (long long)blockIdx.x * kT + threadIdx.x; p < total; p += (long long)gridDim.x * kT) {
    const int n = (int)(p / ((long long)f.h * f.w));
    const int rem = (int)(p - (long long)n * f.h * f.w);
    const int y = rem / f.w, x = rem - y * f.w;
    (void)y;
    (void)x;
    const double dm = 2.0 / (double)f.n * (double)G[p] / E[n];
    const float dy = (float)(dm * s[n]);
    float v[16], g[16];
    ld8(h0 + p * 16, v);
    ld8(h0 + p * 16 + 8, v + 8);
#pragma unroll
    for (int c = 0; c < 16; c++) {
      g[c] = v[c] > 0.0f ? dy * wsm[c] : 0.0f;
      acc[c] += (double)dy * (double)v[c];
    }
    acc[16] += (double)dy;
    st8(g0u + p * 16, g);
    st8(g0u + p * 16 + 8, g + 8);
  }
  for (int c = 0; c < 17; c++) {
    const double t = block_sum_d(acc[c], sm);
    if (threadIdx.x == 0) part[blockIdx.x * 17 + c] = (float)t;
  }
}

// Weight gradient of one 3x3 layer: dW[tap][co][ci] = sum_p g[p][co] x[p + tap][ci]
// (x zero outside the image), db[co] = sum_p g[p][co]. blockIdx.y = tap (9 =
// bias); each CTA sums its pixel tiles; partial[blockIdx.x][...] in W layout.
template <int CIN, int COUT>
__global__ void __launch_bounds__(kT) k_wgrad(const bf16 *x, const bf16 *g, int n, int h, int w, float *partial) {
  constexpr int NO = CIN * COUT, PER = (NO + kT - 1) / kT, LEN = 9 * NO + COUT;
  __shared__ __align__(16) bf16 gs[kWgTile * COUT];
  __shared__ __align__(16) bf16 xs[kWgTile * CIN];
  const int tap = blockIdx.y;
  const int dy = tap / 3 - 1, dx = tap % 3 - 1;
  const int tx = (w + 15) / 16, ty = (h + 7) / 8;
  const int tiles = n * tx * ty;
  float acc[PER];
#pragma unroll
  for (int k = 0; k < PER; k++) acc[k] = 0.0f;
  for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int img = t / (tx * ty), rem = t - img * tx * ty;
    const int y0 = (rem / tx) * 8, x0 = (rem % tx) * 16;
    __syncthreads();
    for (int v = threadIdx.x; v < kWgTile * (COUT / 8); v += kT) {
      const int p = v / (COUT / 8), cg = v % (COUT / 8);
      const int y = y0 + p / 16, xx = x0 + p % 16;
      uint4 val = make_uint4(0, 0, 0, 0);
      if (y < h && xx < w) val = *reinterpret_cast<const uint4 *>(g + (((long long)img * h + y) * w + xx) * COUT + cg * 8);
      *reinterpret_cast<uint4 *>(gs + p * COUT + cg * 8) = val;
    }
    if (tap < 9) {
      for (int v = threadIdx.x; v < kWgTile * (CIN / 8); v += kT) {
        const int p = v / (CIN / 8), cg = v % (CIN / 8);
        const int y = y0 + p / 16 + dy, xx = x0 + p % 16 + dx;
        uint4 val = make_uint4(0, 0, 0, 0);
        if (y >= 0 && y < h && xx >= 0 && xx < w && y0 + p / 16 < h && x0 + p % 16 < w)
          val = *reinterpret_cast<const uint4 *>(x + (((long long)img * h + y) * w + xx) * CIN + cg * 8);
        *reinterpret_cast<uint4 *>(xs + p * CIN + cg * 8) = val;
      }
    }
    __syncthreads();
    if (tap < 9) {
#pragma unroll
      for (int k = 0; k < PER; k++) {
        const int o = threadIdx.x + k * kT;
        if (o < NO) {
          const int co = o / CIN, ci = o - co * CIN;
          float a = acc[k];
          for (int p = 0; p < kWgTile; p++) a += __bfloat162float(gs[p * COUT + co]) * __bfloat162float(xs[p * CIN + ci]);
          acc[k] = a;
        }
      }
    } else if (threadIdx.x < COUT) {
      float a = acc[0];
      for (int p = 0; p < kWgTile; p++) a += __bfloat162float(gs[p * COUT + threadIdx.x]);
      acc[0] = a;
    }
  }
  float *out = partial + (size_t)blockIdx.x * LEN;
  if (tap < 9) {
#pragma unroll
    for (int k = 0; k < PER; k++) {
      const int o = threadIdx.x + k * kT;
      if (o < NO) out[tap * NO + o] = acc[k];
    }
  } else if (threadIdx.x < COUT) {
    out[9 * NO + threadIdx.x] = acc[0];
  }
}

// grad[i] = sum_k partial[k * len + i], k in order.
__global__ void k_sum_parts(const float *partial, int nparts, int len, float *grad) {
  for (int i = blockIdx.x * kT + threadIdx.x; i < len; i += gridDim.x * kT) {
    float t = 0.0f;
    for (int k = 0; k < nparts; k++) t += partial[(size_t)k * len + i];
    grad[i] = t;
  }
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, int np, float lr_t, float b1, float b2,
                       float eps) {
  for (int i = blockIdx.x * kT + threadIdx.x; i < np; i += gridDim.x * kT) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr_t * mi / (sqrtf(vi) + eps);
  }
}

// BF16 copies of one layer's weights: forward [9][cout][cin] and, for the
// input gradient, flipped and transposed [9][cin][cout] with tap' = 8 - tap.
__global__ void k_prep(const float *W, int cin, int cout, bf16 *wf, bf16 *wt) {
  const int total = 9 * cin * cout;
  for (int i = blockIdx.x * kT + threadIdx.x; i < total; i += gridDim.x * kT) {
    const int tap = i / (cin * cout), rem = i - tap * cin * cout;
    const int co = rem / cin, ci = rem - co * cin;
    const bf16 v = __float2bfloat16_rn(W[i]);
    wf[i] = v;
    wt[(8 - tap) * cin * cout + ci * cout + co] = v;
  }
}

int blocks_for(long long work) {
  long long b = (work + kT - 1) / kT;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw Error(E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// SplitMix64 stream for the weight initialisation.
struct Rng {
  unsigned long long s;
  unsigned long long next() {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double u01() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
  double normal() { return sqrt(-2.0 * log(u01())) * cos(6.283185307179586 * u01()); }
};

}  // namespace

struct Net::Impl {
  float *params = nullptr, *grads = nullptr, *am = nullptr, *av = nullptr;
  bf16 *wbuf = nullptr;
  bf16 *wf[kLayers] = {}, *wt[kLayers] = {};
  bool prepped = false;
  int step = 0;
  // activations for (an, ah, aw)
  int an = 0, ah = 0, aw = 0;
  char *act = nullptr;
  bf16 *x0, *e0, *u0, *h0, *p1, *a1, *e1, *u1, *h1, *p2, *a2, *e2, *u2, *h2, *p3, *a3, *h3;
  bf16 *g0u, *du0, *ge0, *g1u, *du1, *ge1, *ga1, *dp1, *g2u, *du2, *ge2, *ga2, *dp2, *g3b, *ga3, *dp3;
  float *pred = nullptr, *gbuf = nullptr, *wpart = nullptr, *opart = nullptr;
  double *dscal = nullptr;  // s[n], E[n], loss, partials
  int zblk = 0;

  ~Impl() {
    cudaFree(params);
    cudaFree(wbuf);
    cudaFree(act);
  }

  void ensure(int n, int h, int w) {
    if (n == an && h == ah && w == aw) return;
    if (h % 8 || w % 8 || h < 8 || w < 8 || n < 1) throw Error(E_ARG, "learned preconditioner: h and w must be multiples of 8");
    cudaFree(act);
    act = nullptr;
    const long long P0 = (long long)n * h * w, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
    struct B {
      bf16 **p;
      long long elems;
    };
    std::vector<B> list = {
        {&x0, P0 * 16}, {&e0, P0 * 16}, {&u0, P0 * 16}, {&h0, P0 * 16}, {&p1, P1 * 16}, {&a1, P1 * 32},
        {&e1, P1 * 32}, {&u1, P1 * 32}, {&h1, P1 * 16}, {&p2, P2 * 32}, {&a2, P2 * 64}, {&e2, P2 * 64},
        {&u2, P2 * 64}, {&h2, P2 * 32}, {&p3, P3 * 64}, {&a3, P3 * 64}, {&h3, P3 * 64}, {&g0u, P0 * 16},
        {&du0, P0 * 16}, {&ge0, P0 * 16}, {&g1u, P1 * 16}, {&du1, P1 * 32}, {&ge1, P1 * 32}, {&ga1, P1 * 32},
        {&dp1, P1 * 16}, {&g2u, P2 * 32}, {&du2, P2 * 64}, {&ge2, P2 * 64}, {&ga2, P2 * 64}, {&dp2, P2 * 32},
        {&g3b, P3 * 64}, {&ga3, P3 * 64}, {&dp3, P3 * 64}};
    size_t bytes = 0;
    for (auto &b : list) bytes += ((size_t)b.elems * 2 + 255) / 256 * 256;
    zblk = (int)std::max<long long>(1, std::min<long long>(std::min<long long>(1024, 148 * 8 / n),
                                                            (h * (long long)w + kT - 1) / kT));
    const size_t pred_b = ((size_t)P0 * 4 + 255) / 256 * 256;
    int maxlen = 0;
    for (int l = 0; l < kLayers; l++) maxlen = std::max(maxlen, 9 * kDefs[l].cin * kDefs[l].cout + kDefs[l].cout);
    const size_t wpart_b = ((size_t)kWgX * maxlen * 4 + 255) / 256 * 256;
    const size_t opart_b = ((size_t)148 * 16 * 17 * 4 + 255) / 256 * 256;
    const size_t dscal_b = ((size_t)(2 * n + 1 + 2 * n * zblk) * 8 + 255) / 256 * 256;
    check(cudaMalloc(&act, bytes + 2 * pred_b + wpart_b + opart_b + dscal_b), "learned preconditioner buffers");
    char *c = act;
    for (auto &b : list) {
      *b.p = reinterpret_cast<bf16 *>(c);
      c += ((size_t)b.elems * 2 + 255) / 256 * 256;
    }
    pred = reinterpret_cast<float *>(c);
    c += pred_b;
    gbuf = reinterpret_cast<float *>(c);
    c += pred_b;
    wpart = reinterpret_cast<float *>(c);
    c += wpart_b;
    opart = reinterpret_cast<float *>(c);
    c += opart_b;
    dscal = reinterpret_cast<double *>(c);
    an = n;
    ah = h;
    aw = w;
  }
};

int Net::num_params() { return offs().total; }

Net::Net(unsigned long long seed) : m_(new Impl) {
  const Offsets &o = offs();
  check(cudaMalloc(&m_->params, (size_t)4 * o.total * 4), "learned preconditioner parameters");
  m_->grads = m_->params + o.total;
  m_->am = m_->grads + o.total;
  m_->av = m_->am + o.total;
  check(cudaMemset(m_->params, 0, (size_t)4 * o.total * 4), "learned preconditioner parameters");
  size_t wel = 0;
  for (int l = 0; l < kLayers; l++) wel += 9 * kDefs[l].cin * kDefs[l].cout;
  check(cudaMalloc(&m_->wbuf, wel * 2 * 2 + 512), "learned preconditioner weights");
  bf16 *p = m_->wbuf;
  for (int l = 0; l < kLayers; l++) {
    const int e = 9 * kDefs[l].cin * kDefs[l].cout;
    m_->wf[l] = p;
    p += e;
    m_->wt[l] = p;
    p += e;
  }
  // He-normal weights, zero biases, zero output layer (an untrained net is Jacobi)
  std::vector<float> h(o.total, 0.0f);
  Rng rng{seed};
  for (int l = 0; l < kLayers; l++) {
    const double sd = sqrt(2.0 / (9.0 * kDefs[l].cin));
    for (int i = 0; i < 9 * kDefs[l].cin * kDefs[l].cout; i++) h[o.w[l] + i] = (float)(sd * rng.normal());
  }
  set_params(h.data());
}

Net::~Net() { delete m_; }

void Net::get_params(float *host) const {
  check(cudaMemcpy(host, m_->params, (size_t)offs().total * 4, cudaMemcpyDeviceToHost), "get params");
}
void Net::get_grads(float *host) const {
  check(cudaMemcpy(host, m_->grads, (size_t)offs().total * 4, cudaMemcpyDeviceToHost), "get grads");
}
void Net::set_params(const float *host) {
  check(cudaMemcpy(m_->params, host, (size_t)offs().total * 4, cudaMemcpyHostToDevice), "set params");
  check(cudaMemset(m_->am, 0, (size_t)2 * offs().total * 4), "reset adam");
  m_->step = 0;
  m_->prepped = false;
}

namespace {
void conv(const bf16 *x, const bf16 *w, int n, int h, int wd, int cin, int cout, const float *bias, const bf16 *mask,
          bf16 *y, int mode, cudaStream_t s) {
  cudaError_t e = cnn::conv3x3(x, w, n, h, wd, cin, cout, bias, mask, y, mode, cnn::error_word(), s);
  check(e, "learned preconditioner conv3x3");
}
}  // namespace

// Forward pass through h0 (features, encoder, decoder). Returns nothing; the
// output layer is applied by the callers.
static void forward(Net::Impl &m, const Fields &f, cudaStream_t s, long long &launches) {
  const Offsets &o = offs();
  if (!m.prepped) {
    for (int l = 0; l < kLayers; l++)
      k_prep<<<blocks_for(9 * kDefs[l].cin * kDefs[l].cout), kT, 0, s>>>(m.params + o.w[l], kDefs[l].cin,
                                                                         kDefs[l].cout, m.wf[l], m.wt[l]);
    launches += kLayers;
    m.prepped = true;
  }
  const int n = f.n, h = f.h, w = f.w;
  double *spart = m.dscal + 2 * n + 1;
  k_zsq<<<dim3(m.zblk, n), kT, 0, s>>>(f, spart);
  k_scale<<<(n + 63) / 64, 64, 0, s>>>(spart, m.zblk, h * w, m.dscal, n);
  k_features<<<blocks_for((long long)n * h * w), kT, 0, s>>>(f, m.dscal, m.x0);
  auto B = [&](int l) { return m.params + o.b[l]; };
  const int h1 = h / 2, w1 = w / 2, h2 = h / 4, w2 = w / 4, h3 = h / 8, w3 = w / 8;
  conv(m.x0, m.wf[C0], n, h, w, 16, 16, B(C0), nullptr, m.e0, cnn::CONV_BIAS_RELU, s);
  k_pool<<<blocks_for((long long)n * h1 * w1 * 2), kT, 0, s>>>(m.e0, m.p1, n, h, w, 16);
  conv(m.p1, m.wf[C1A], n, h1, w1, 16, 32, B(C1A), nullptr, m.a1, cnn::CONV_BIAS_RELU, s);
  conv(m.a1, m.wf[C1B], n, h1, w1, 32, 32, B(C1B), nullptr, m.e1, cnn::CONV_BIAS_RELU, s);
  k_pool<<<blocks_for((long long)n * h2 * w2 * 4), kT, 0, s>>>(m.e1, m.p2, n, h1, w1, 32);
  conv(m.p2, m.wf[C2A], n, h2, w2, 32, 64, B(C2A), nullptr, m.a2, cnn::CONV_BIAS_RELU, s);
  conv(m.a2, m.wf[C2B], n, h2, w2, 64, 64, B(C2B), nullptr, m.e2, cnn::CONV_BIAS_RELU, s);
  k_pool<<<blocks_for((long long)n * h3 * w3 * 8), kT, 0, s>>>(m.e2, m.p3, n, h2, w2, 64);
  conv(m.p3, m.wf[C3A], n, h3, w3, 64, 64, B(C3A), nullptr, m.a3, cnn::CONV_BIAS_RELU, s);
  conv(m.a3, m.wf[C3B], n, h3, w3, 64, 64, B(C3B), nullptr, m.h3, cnn::CONV_BIAS_RELU, s);
  k_up_add<<<blocks_for((long long)n * h2 * w2 * 8), kT, 0, s>>>(m.h3, m.e2, m.u2, n, h2, w2, 64);
  conv(m.u2, m.wf[C2U], n, h2, w2, 64, 32, B(C2U), nullptr, m.h2, cnn::CONV_BIAS_RELU, s);
  k_up_add<<<blocks_for((long long)n * h1 * w1 * 4), kT, 0, s>>>(m.h2, m.e1, m.u1, n, h1, w1, 32);
  conv(m.u1, m.wf[C1U], n, h1, w1, 32, 16, B(C1U), nullptr, m.h1, cnn::CONV_BIAS_RELU, s);
  k_up_add<<<blocks_for((long long)n * h * w * 2), kT, 0, s>>>(m.h1, m.e0, m.u0, n, h, w, 16);
  conv(m.u0, m.wf[C0U], n, h, w, 16, 16, B(C0U), nullptr, m.h0, cnn::CONV_BIAS_RELU, s);
  check(cudaGetLastError(), "learned preconditioner forward");
  launches += 19;
}

void Net::apply(const Fields &f, double *out, cudaStream_t s) {
  m_->ensure(f.n, f.h, f.w);
  check(cudaMemsetAsync(cnn::error_word(), 0, sizeof(int), s), "conv error word");
  forward(*m_, f, s, launches_);
  k_out<<<blocks_for((long long)f.n * f.h * f.w), kT, 0, s>>>(f, m_->dscal, m_->h0, m_->params, offs().wout, out,
                                                              f.image, f.pitch, nullptr);
  check(cudaGetLastError(), "learned preconditioner output");
  launches_ += 1;
}

namespace {
template <int CI, int CO>
void wgrad(const bf16 *x, const bf16 *g, int n, int h, int w, float *wpart, float *grad, cudaStream_t s) {
  const int tiles = n * ((w + 15) / 16) * ((h + 7) / 8);
  const int gx = std::min(kWgX, tiles);
  k_wgrad<CI, CO><<<dim3(gx, 10), kT, 0, s>>>(x, g, n, h, w, wpart);
  const int len = 9 * CI * CO + CO;
  k_sum_parts<<<blocks_for(len), kT, 0, s>>>(wpart, gx, len, grad);
}
}  // namespace

double Net::loss_and_grad(const Fields &f, const double *e, int kind, cudaStream_t s) {
  Impl &m = *m_;
  m.ensure(f.n, f.h, f.w);
  check(cudaMemsetAsync(cnn::error_word(), 0, sizeof(int), s), "conv error word");
  forward(m, f, s, launches_);
  const Offsets &o = offs();
  const int n = f.n, h = f.h, w = f.w;
  k_out<<<blocks_for((long long)n * h * w), kT, 0, s>>>(f, m.dscal, m.h0, m.params, o.wout, nullptr, 0, 0, m.pred);
  double *E = m.dscal + n, *loss = m.dscal + 2 * n, *lpart = m.dscal + 2 * n + 1;
  k_diff<<<dim3(m.zblk, n), kT, 0, s>>>(f, m.pred, e, lpart);
  const float *G = m.pred;
  if (kind == LOSS_ANORM) {
    k_anorm<<<dim3(m.zblk, n), kT, 0, s>>>(f, m.pred, e, m.gbuf, lpart);
    G = m.gbuf;
    launches_ += 1;
  }
  k_loss_finish<<<1, 32, 0, s>>>(lpart, m.zblk, n, E, loss);
  const int ob = blocks_for((long long)n * h * w);
  k_out_bwd<<<ob, kT, 0, s>>>(f, m.dscal, E, G, m.h0, m.params, o.wout, m.g0u, m.opart);
  k_sum_parts<<<1, kT, 0, s>>>(m.opart, ob, 17, m.grads + o.wout);
  launches_ += 6;
  const int h1 = h / 2, w1 = w / 2, h2 = h / 4, w2 = w / 4, h3 = h / 8, w3 = w / 8;
  // input gradients (tensor cores, flipped/transposed weights)
  conv(m.g0u, m.wt[C0U], n, h, w, 16, 16, nullptr, nullptr, m.du0, cnn::CONV_PLAIN, s);
  k_upT_mask<<<blocks_for((long long)n * h1 * w1 * 2), kT, 0, s>>>(m.du0, m.h1, m.g1u, n, h, w, 16);
  conv(m.g1u, m.wt[C1U], n, h1, w1, 16, 32, nullptr, nullptr, m.du1, cnn::CONV_PLAIN, s);
  k_upT_mask<<<blocks_for((long long)n * h2 * w2 * 4), kT, 0, s>>>(m.du1, m.h2, m.g2u, n, h1, w1, 32);
  conv(m.g2u, m.wt[C2U], n, h2, w2, 32, 64, nullptr, nullptr, m.du2, cnn::CONV_PLAIN, s);
  k_upT_mask<<<blocks_for((long long)n * h3 * w3 * 8), kT, 0, s>>>(m.du2, m.h3, m.g3b, n, h2, w2, 64);
  conv(m.g3b, m.wt[C3B], n, h3, w3, 64, 64, nullptr, m.a3, m.ga3, cnn::CONV_MASK, s);
  conv(m.ga3, m.wt[C3A], n, h3, w3, 64, 64, nullptr, nullptr, m.dp3, cnn::CONV_PLAIN, s);
  k_add_poolT_mask<<<blocks_for((long long)n * h2 * w2 * 8), kT, 0, s>>>(m.du2, m.dp3, m.e2, m.ge2, n, h2, w2, 64);
  conv(m.ge2, m.wt[C2B], n, h2, w2, 64, 64, nullptr, m.a2, m.ga2, cnn::CONV_MASK, s);
  conv(m.ga2, m.wt[C2A], n, h2, w2, 64, 32, nullptr, nullptr, m.dp2, cnn::CONV_PLAIN, s);
  k_add_poolT_mask<<<blocks_for((long long)n * h1 * w1 * 4), kT, 0, s>>>(m.du1, m.dp2, m.e1, m.ge1, n, h1, w1, 32);
  conv(m.ge1, m.wt[C1B], n, h1, w1, 32, 32, nullptr, m.a1, m.ga1, cnn::CONV_MASK, s);
  conv(m.ga1, m.wt[C1A], n, h1, w1, 32, 16, nullptr, nullptr, m.dp1, cnn::CONV_PLAIN, s);
  k_add_poolT_mask<<<blocks_for((long long)n * h * w * 2), kT, 0, s>>>(m.du0, m.dp1, m.e0, m.ge0, n, h, w, 16);
  launches_ += 16;
  // weight gradients (CUDA cores, fixed-order partial sums)
  float *WG = m.grads;
  wgrad<16, 16>(m.u0, m.g0u, n, h, w, m.wpart, WG + o.w[C0U], s);
  wgrad<32, 16>(m.u1, m.g1u, n, h1, w1, m.wpart, WG + o.w[C1U], s);
  wgrad<64, 32>(m.u2, m.g2u, n, h2, w2, m.wpart, WG + o.w[C2U], s);
  wgrad<64, 64>(m.a3, m.g3b, n, h3, w3, m.wpart, WG + o.w[C3B], s);
  wgrad<64, 64>(m.p3, m.ga3, n, h3, w3, m.wpart, WG + o.w[C3A], s);
  wgrad<64, 64>(m.a2, m.ge2, n, h2, w2, m.wpart, WG + o.w[C2B], s);
  wgrad<32, 64>(m.p2, m.ga2, n, h2, w2, m.wpart, WG + o.w[C2A], s);
  wgrad<32, 32>(m.a1, m.ge1, n, h1, w1, m.wpart, WG + o.w[C1B], s);
  wgrad<16, 32>(m.p1, m.ga1, n, h1, w1, m.wpart, WG + o.w[C1A], s);
  wgrad<16, 16>(m.x0, m.ge0, n, h, w, m.wpart, WG + o.w[C0], s);
  check(cudaGetLastError(), "learned preconditioner backward");
  launches_ += 20;
  double L = 0.0;
  check(cudaMemcpyAsync(&L, loss, 8, cudaMemcpyDeviceToHost, s), "loss readback");
  check(cudaStreamSynchronize(s), "learned preconditioner step");
  int err = 0;
  check(cudaMemcpy(&err, cnn::error_word(), 4, cudaMemcpyDeviceToHost), "conv error word");
  if (err) throw Error(E_TIMEOUT, "learned preconditioner: a convolution pipeline wait expired");
  return L;
}

void Net::adam(double lr, cudaStream_t s) {
  Impl &m = *m_;
  const int np = offs().total;
  m.step++;
  const double b1 = 0.9, b2 = 0.999;
  const double lr_t = lr * sqrt(1.0 - pow(b2, m.step)) / (1.0 - pow(b1, m.step));
  k_adam<<<blocks_for(np), kT, 0, s>>>(m.params, m.grads, m.am, m.av, np, (float)lr_t, (float)b1, (float)b2, 1e-8f);
  check(cudaGetLastError(), "adam");
  launches_ += 1;
  m.prepped = false;
}

}  // namespace lmg
}  // namespace opsb
