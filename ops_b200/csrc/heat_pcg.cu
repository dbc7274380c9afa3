// Device-resident Jacobi-PCG for the TeaLeaf 2D heat operator; interface and
// algorithm notes in heat_pcg.h.
//
// Per iteration (tea_leaf_cg.cpp:103-214, one kernel per reference routine):
//   k_w   w = A p, pw = p.w                  -> last block: alpha = rro / pw
//   k_ur  u += alpha p, r -= alpha w, z = Mi r, rz = r.z
//                                            -> last block: beta, rro, stop test
//   k_p   p = beta p + z
// The arithmetic of every cell is the reference's, in its order (this file
// builds without FMA contraction). Grid sums finish in a fixed order (each
// block's partial, then the last block to arrive adds the partials by block
// index), so a solve is bit-reproducible run to run. Once the stop test has
// fired every later kernel returns at entry, so a chunk of iterations that
// runs past convergence costs only its launch latency.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "heat_pcg.h"
#include "runtime.h"

namespace opsb {
namespace heat {

namespace {

constexpr int BX = 128, BY = 2, NT = BX * BY, kWarps = NT / 32;
constexpr int kMaxBlocks = 4096;
constexpr int kChunk = 16;          // iterations per replayed graph
// Grids are one wave of kResident blocks per SM; every kernel is held to the
// registers that let kResident blocks stay resident (a kernel over budget
// would run its grid in 1 1/3 waves).
constexpr int kResident = 8;
constexpr int kTargetBlocks = 148 * kResident;

struct Scalars {
  double rro, rro_prev, pw, alpha, beta;
  double err, stop, ref, rr, rr0;
  int done;       // 0 running, 1 converged, 2 iteration limit, 3 reliable update due,
                  // 4 FCG lost positive curvature, 5 FCG restart (||r|| not halved over the window)
  int iters;
  int max_iters;
  int first;
  // FCG restart test on the device (replayed chunks): ||r|| of the last
  // iterations since the last (re)start, `window` 0 when the test is off
  int window, hcount;
  double hist[64];
};

// Stopping quantity of k_ur.
enum { STOP_TEALEAF = 0,  // sqrt|r.z| < eps ||r0|| (tea_solve.cpp:349-355)
       STOP_TRUE = 1,     // ||r|| < eps ||r0||
       STOP_RELIABLE = 2  // inner FP32 loop: estimate test, or a decade of decrease since the last update
};

struct Geom {
  int nx, ny;
  long long pitch;
};

__device__ __forceinline__ int tid_() { return threadIdx.x + threadIdx.y * BX; }

// Sum over the block; the result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *sm) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int t = tid_(), lane = t & 31, wid = t >> 5;
  __syncthreads();
  if (lane == 0) sm[wid] = v;
  __syncthreads();
  v = 0.0;
  if (wid == 0) {
    v = lane < kWarps ? sm[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// Stores the block's partials (NV values, part[NV * block + k]); true in
// every thread of the last block to arrive.
template <int NV>
__device__ __forceinline__ bool publish(const double (&v)[NV], double *part, unsigned *cnt, double *sm, int *last) {
  const int nb = gridDim.x * gridDim.y, bid = blockIdx.x + blockIdx.y * gridDim.x;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    const double b = block_sum(v[k], sm);
    if (tid_() == 0) part[NV * bid + k] = b;
  }
  if (tid_() == 0) {
    __threadfence();
    const unsigned t = atomicAdd(cnt, 1u);
    *last = (t == (unsigned)(nb - 1));
  }
  __syncthreads();
  return *last != 0;
}

// Last block only: partial k of every block added in block order; valid in
// thread 0. The caller resets the arrival counter once all totals are taken.
template <int NV>
__device__ __forceinline__ double grid_total(const double *part, int k, double *sm) {
  __threadfence();
  const int nb = gridDim.x * gridDim.y;
  double v = 0.0;
  for (int b = tid_(); b < nb; b += NT) v += __ldcg(part + NV * b + k);
  return block_sum(v, sm);
}

// tea_leaf_common_kernels.h (the 5-point operator shared by the CG kernels).
template <class T>
__device__ __forceinline__ T smvp(const T *__restrict__ Kx, const T *__restrict__ Ky, const T *__restrict__ u,
                                  long long i, long long P, T rx, T ry) {
  const T kx0 = Kx[i], kx1 = Kx[i + 1], ky0 = Ky[i], ky1 = Ky[i + P];
  return (T(1) + ry * (ky1 + ky0) + rx * (kx1 + kx0)) * u[i] - ry * (ky1 * u[i + P] + ky0 * u[i - P]) -
         rx * (kx1 * u[i + 1] + kx0 * u[i - 1]);
}

#define HEAT_CELLS(g)                                                                          \
  for (int y = blockIdx.y * BY + threadIdx.y; y < (g).ny; y += gridDim.y * BY)                 \
    for (int x = blockIdx.x * BX + threadIdx.x; x < (g).nx; x += gridDim.x * BX)

// tea_leaf_cg_calc_w_reduce_kernel (tea_leaf_cg_kernels.h:8) + alpha = rro/pw.
template <class T>
__global__ void __launch_bounds__(NT, kResident) k_w(Geom g, const T *__restrict__ Kx, const T *__restrict__ Ky,
                                          const T *__restrict__ p, T *__restrict__ w, T rx, T ry, Scalars *s,
                                          double *part, unsigned *cnt) {
  __shared__ double sm[kWarps];
  __shared__ int last;
  if (s->done) return;
  double acc[1] = {0.0};
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    const T wv = smvp(Kx, Ky, p, i, g.pitch, rx, ry);
    w[i] = wv;
    acc[0] = acc[0] + (double)wv * (double)p[i];
  }
  if (publish<1>(acc, part, cnt, sm, &last)) {
    const double t = grid_total<1>(part, 0, sm);
    if (tid_() == 0) {
      s->pw = t;
      s->alpha = s->rro / t;
      *cnt = 0u;
    }
  }
}

// tea_leaf_axpy_kernel on u and r, tea_leaf_zeqxty_kernel (z = Mi r) and
// tea_leaf_dot_kernel (r.z), or tea_leaf_cg_calc_ur_r_reduce_kernel (r.r)
// without preconditioner; then beta = rrn/rro and the stop test.
template <class T, bool PREC, int STOP>
__global__ void __launch_bounds__(NT, kResident) k_ur(Geom g, T *__restrict__ u, const T *__restrict__ p, T *__restrict__ r,
                                           const T *__restrict__ w, const T *__restrict__ Mi, T *__restrict__ z,
                                           Scalars *s, double *part, unsigned *cnt) {
  constexpr int NV = (STOP == STOP_TRUE && PREC) ? 2 : 1;
  __shared__ double sm[kWarps];
  __shared__ int last;
  if (s->done) return;
  const T alpha = (T)s->alpha;
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) acc[k] = 0.0;
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    u[i] = u[i] + alpha * p[i];
    const T rv = r[i] - alpha * w[i];
    r[i] = rv;
    if (PREC) {
      const T zv = Mi[i] * rv;
      z[i] = zv;
      acc[0] = acc[0] + (double)rv * (double)zv;
    } else {
      acc[0] = acc[0] + (double)rv * (double)rv;
    }
    if (NV == 2) acc[NV - 1] = acc[NV - 1] + (double)rv * (double)rv;
  }
  if (publish<NV>(acc, part, cnt, sm, &last)) {
    const double t = grid_total<NV>(part, 0, sm);
    const double rr = NV == 2 ? grid_total<NV>(part, NV - 1, sm) : t;
    if (tid_() == 0) {
      s->rro_prev = s->rro;
      s->beta = t / s->rro;
      s->rro = t;
      s->iters = s->iters + 1;
      const double err = STOP == STOP_TRUE ? sqrt(fabs(rr)) : sqrt(fabs(t));
      s->err = err;
      if (fabs(err) < s->stop) s->done = 1;
      else if (STOP == STOP_RELIABLE && err < s->ref) s->done = 3;
      else if (s->iters >= s->max_iters) s->done = 2;
      *cnt = 0u;
    }
  }
}

// tea_leaf_axpby_kernel with alpha = beta, beta = 1 (tea_leaf_cg.cpp:188-214).
template <class T>
__global__ void __launch_bounds__(NT, kResident) k_p(Geom g, T *__restrict__ p, const T *__restrict__ z, const Scalars *s) {
  if (s->done) return;
  const T beta = (T)s->beta;
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    p[i] = beta * p[i] + z[i];
  }
}

// tea_leaf_common_residual_kernel + tea_leaf_norm2_kernel (tea_leaf_common.cpp:160-211):
// r = u0 - A u, rr = r.r. The first call of a solve fixes ||r0|| and the
// stop threshold eps * ||r0|| (tea_solve.cpp:105-114); later calls test against it.
__global__ void __launch_bounds__(NT, kResident) k_resid(Geom g, const double *__restrict__ Kx, const double *__restrict__ Ky,
                                              const double *__restrict__ u, const double *__restrict__ u0,
                                              double *__restrict__ r, double rx, double ry, double eps, Scalars *s,
                                              double *part, unsigned *cnt) {
  __shared__ double sm[kWarps];
  __shared__ int last;
  double acc[1] = {0.0};
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    const double smv = smvp(Kx, Ky, u, i, g.pitch, rx, ry);
    const double rv = u0[i] - smv;
    r[i] = rv;
    acc[0] = acc[0] + rv * rv;
  }
  if (publish<1>(acc, part, cnt, sm, &last)) {
    const double t = grid_total<1>(part, 0, sm);
    if (tid_() == 0) {
      s->rr = t;
      const double nrm = sqrt(fabs(t));
      if (s->first) {
        s->rr0 = t;
        s->stop = eps * nrm;
        s->first = 0;
      }
      s->err = nrm;
      s->done = (fabs(nrm) < s->stop) ? 1 : 0;
      *cnt = 0u;
    }
  }
}

// cg_init (tea_leaf_cg.cpp:53-101): z = Mi r (or none), p = z (or r), rro = r.p.
template <bool PREC>
__global__ void __launch_bounds__(NT, kResident) k_init(Geom g, const double *__restrict__ r, const double *__restrict__ Mi,
                                             double *__restrict__ z, double *__restrict__ p, int max_iters,
                                             Scalars *s, double *part, unsigned *cnt) {
  __shared__ double sm[kWarps];
  __shared__ int last;
  double acc[1] = {0.0};
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    const double rv = r[i];
    double pv = rv;
    if (PREC) {
      pv = Mi[i] * rv;
      z[i] = pv;
    }
    p[i] = pv;
    acc[0] = acc[0] + rv * pv;
  }
  if (publish<1>(acc, part, cnt, sm, &last)) {
    const double t = grid_total<1>(part, 0, sm);
    if (tid_() == 0) {
      s->rro = t;
      s->iters = 0;
      s->max_iters = max_iters;
      s->done = 0;
      *cnt = 0u;
    }
  }
}

// Reliable update of the FP32 loop (Sleijpen and van der Vorst 1996, "Reliable
// updated residuals in hybrid Bi-CG methods"): the recursive FP32 residual is
// replaced by the FP64 residual r64 = u0 - A u, z32 = Mi32 r32, and the search
// direction is kept: beta = rz_new / rz_prev, followed by k_p. The first call
// starts the loop (beta = 0 with p32 = 0, so p = z) and fixes the estimate
// threshold eps * sqrt(rz0); `scale` tightens it after an estimate that the
// FP64 check did not confirm. The next update is due once sqrt(rz) has fallen
// by `delta`.
template <bool PREC>
__global__ void __launch_bounds__(NT, kResident) k_reinit32(Geom g, Geom g32, const double *__restrict__ r64,
                                                 float *__restrict__ r, const float *__restrict__ Mi,
                                                 float *__restrict__ z, int first, double eps, double scale,
                                                 double delta, int max_iters, Scalars *s, double *part,
                                                 unsigned *cnt) {
  __shared__ double sm[kWarps];
  __shared__ int last;
  double acc[1] = {0.0};
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    const long long j = (long long)y * g32.pitch + x;
    const float rv = (float)r64[i];
    r[j] = rv;
    float zv = rv;
    if (PREC) {
      zv = Mi[j] * rv;
      z[j] = zv;
    }
    acc[0] = acc[0] + (double)rv * (double)zv;
  }
  if (publish<1>(acc, part, cnt, sm, &last)) {
    const double t = grid_total<1>(part, 0, sm);
    if (tid_() == 0) {
      if (first) {
        s->rr0 = t;
        s->iters = 0;
        s->max_iters = max_iters;
        s->beta = 0.0;
      } else {
        s->beta = t / s->rro_prev;
      }
      s->stop = eps * scale * sqrt(fabs(s->rr0));
      s->ref = delta * sqrt(fabs(t));
      s->rro = t;
      s->done = 0;
      *cnt = 0u;
    }
  }
}

// Reliable update, FP64 side: u += e, e = 0.
__global__ void __launch_bounds__(NT, kResident) k_update(Geom g, Geom g32, double *__restrict__ u, float *__restrict__ e) {
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    const long long j = (long long)y * g32.pitch + x;
    u[i] = u[i] + (double)e[j];
    e[j] = 0.0f;
  }
}

// FP32 copies of Kx, Ky, Mi over the interior and its one-cell ring.
__global__ void __launch_bounds__(NT, kResident) k_to_float(Geom g, Geom g32, const double *__restrict__ a,
                                                 const double *__restrict__ b, const double *__restrict__ c,
                                                 float *__restrict__ fa, float *__restrict__ fb,
                                                 float *__restrict__ fc) {
  for (int y = blockIdx.y * BY + threadIdx.y - 1; y < g.ny + 1; y += gridDim.y * BY)
    for (int x = blockIdx.x * BX + threadIdx.x - 1; x < g.nx + 1; x += gridDim.x * BX) {
      const long long i = (long long)y * g.pitch + x, j = (long long)y * g32.pitch + x;
      fa[j] = (float)a[i];
      fb[j] = (float)b[i];
      if (c) fc[j] = (float)c[i];
    }
}


// ---- flexible CG (Notay 2000, FCG with one-step truncation) ----------------
// k_fw: w = A p, pw = p.w, pr = p.r -> alpha = pr / pw; a non-positive pw
// (the preconditioned direction lost positive curvature) stops with done = 4.
__global__ void __launch_bounds__(NT, kResident) k_fw(Geom g, const double *__restrict__ Kx, const double *__restrict__ Ky,
                                           const double *__restrict__ p, const double *__restrict__ r,
                                           double *__restrict__ w, double rx, double ry, Scalars *s, double *part,
                                           unsigned *cnt) {
  __shared__ double sm[kWarps];
  __shared__ int last;
  if (s->done) return;
  double acc[2] = {0.0, 0.0};
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    const double wv = smvp(Kx, Ky, p, i, g.pitch, rx, ry);
    w[i] = wv;
    acc[0] = acc[0] + wv * p[i];
    acc[1] = acc[1] + p[i] * r[i];
  }
  if (publish<2>(acc, part, cnt, sm, &last)) {
    const double pw = grid_total<2>(part, 0, sm);
    const double pr = grid_total<2>(part, 1, sm);
    if (tid_() == 0) {
      s->pw = pw;
      if (pw > 0.0) s->alpha = pr / pw;
      else s->done = 4;
      *cnt = 0u;
    }
  }
}

// u += alpha p, r -= alpha w, rr = r.r; stop when ||r|| < eps ||r0||.
__global__ void __launch_bounds__(NT, kResident) k_fupd(Geom g, double *__restrict__ u, const double *__restrict__ p,
                                             double *__restrict__ r, const double *__restrict__ w, Scalars *s,
                                             double *part, unsigned *cnt) {
  __shared__ double sm[kWarps];
  __shared__ int last;
  if (s->done) return;
  const double alpha = s->alpha;
  double acc[1] = {0.0};
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    u[i] = u[i] + alpha * p[i];
    const double rv = r[i] - alpha * w[i];
    r[i] = rv;
    acc[0] = acc[0] + rv * rv;
  }
  if (publish<1>(acc, part, cnt, sm, &last)) {
    const double t = grid_total<1>(part, 0, sm);
    if (tid_() == 0) {
      s->rr = t;
      s->err = sqrt(t);
      s->iters = s->iters + 1;
      if (s->err < s->stop) s->done = 1;
      else if (s->iters >= s->max_iters) s->done = 2;
      if (s->done == 0 && s->window > 0) {  // the same test the host loop applies
        const int k = s->hcount;
        s->hist[k & 63] = s->err;
        s->hcount = k + 1;
        if (k + 1 > s->window && s->err > 0.5 * s->hist[(k - s->window) & 63]) s->done = 5;
      }
      *cnt = 0u;
    }
  }
}

// beta = -(z.w) / pw.
__global__ void __launch_bounds__(NT, kResident) k_fzw(Geom g, const double *__restrict__ z, const double *__restrict__ w,
                                            Scalars *s, double *part, unsigned *cnt) {
  __shared__ double sm[kWarps];
  __shared__ int last;
  if (s->done) return;  // the solve stopped earlier in a replayed chunk
  double acc[1] = {0.0};
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    acc[0] = acc[0] + z[i] * w[i];
  }
  if (publish<1>(acc, part, cnt, sm, &last)) {
    const double t = grid_total<1>(part, 0, sm);
    if (tid_() == 0) {
      s->beta = -t / s->pw;
      *cnt = 0u;
    }
  }
}

// p = z + beta p, or p = z on a restart.
__global__ void __launch_bounds__(NT, kResident) k_fp(Geom g, double *__restrict__ p, const double *__restrict__ z,
                                           const Scalars *s, int restart) {
  if (!restart && s->done) return;  // the solve stopped earlier in a replayed chunk
  const double beta = restart ? 0.0 : s->beta;
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    p[i] = restart ? z[i] : z[i] + beta * p[i];
  }
}

// z = Mi r (Jacobi).
__global__ void __launch_bounds__(NT, kResident) k_jacobi(Geom g, const double *__restrict__ Mi, const double *__restrict__ r,
                                               double *__restrict__ z) {
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    z[i] = Mi[i] * r[i];
  }
}

// tea_leaf_common_init_diag_init_kernel (tea_leaf_common_kernels.h:38):
// Mi = 1 / (1 + ry (Ky(0,1) + Ky(0,0)) + rx (Kx(1,0) + Kx(0,0))) on the interior.
__global__ void __launch_bounds__(NT, kResident) k_diag(Geom g, const double *__restrict__ Kx, const double *__restrict__ Ky,
                                             double rx, double ry, double *__restrict__ Mi) {
  HEAT_CELLS(g) {
    const long long i = (long long)y * g.pitch + x;
    Mi[i] = 1.0 / (1.0 + ry * (Ky[i + g.pitch] + Ky[i]) + rx * (Kx[i + 1] + Kx[i]));
  }
}

// ---- 3D: the 7-point heat operator ------------------------------------------
// Interior cells (x, y, z) at i = z * plane + y * pitch + x from the first
// interior cell; Kz[i] is the face between z-1 and z (as Kx, Ky in 2D).
// The pointwise CG kernels run on the padded volume as a flat array (the
// solver's own fields are zero on every halo cell), so only the operator,
// the residual and the diagonal need these.
struct Geom3 {
  int nx, ny, nz;
  long long pitch, plane;
};

#define HEAT_CELLS3(g)                                                                                        \
  for (int row = blockIdx.y * BY + threadIdx.y, y = row % (g).ny, z = row / (g).ny; row < (g).ny * (g).nz;   \
       row += gridDim.y * BY, y = row % (g).ny, z = row / (g).ny)                                            \
    for (int x = blockIdx.x * BX + threadIdx.x; x < (g).nx; x += gridDim.x * BX)

template <class T>
__device__ __forceinline__ T smvp3(const T *__restrict__ Kx, const T *__restrict__ Ky, const T *__restrict__ Kz,
                                   const T *__restrict__ u, long long i, long long P, long long Q, T rx, T ry, T rz) {
  const T kx0 = Kx[i], kx1 = Kx[i + 1], ky0 = Ky[i], ky1 = Ky[i + P], kz0 = Kz[i], kz1 = Kz[i + Q];
  return (T(1) + rz * (kz1 + kz0) + ry * (ky1 + ky0) + rx * (kx1 + kx0)) * u[i] - rz * (kz1 * u[i + Q] + kz0 * u[i - Q]) -
         ry * (ky1 * u[i + P] + ky0 * u[i - P]) - rx * (kx1 * u[i + 1] + kx0 * u[i - 1]);
}

// w = A p on the interior, pw = p.w -> alpha = rro / pw (k_w in 3D; FP64, or
// FP32 for the mixed solver's inner iterations).
template <class T>
__global__ void __launch_bounds__(NT, kResident) k_w3(Geom3 g, const T *__restrict__ Kx, const T *__restrict__ Ky,
                                                     const T *__restrict__ Kz, const T *__restrict__ p,
                                                     T *__restrict__ w, T rx, T ry, T rz, Scalars *s, double *part,
                                                     unsigned *cnt) {
  __shared__ double sm[kWarps];
  __shared__ int last;
  if (s->done) return;
  double acc[1] = {0.0};
  HEAT_CELLS3(g) {
    const long long i = (long long)z * g.plane + (long long)y * g.pitch + x;
    const T wv = smvp3<T>(Kx, Ky, Kz, p, i, g.pitch, g.plane, rx, ry, rz);
    w[i] = wv;
    acc[0] = acc[0] + (double)wv * (double)p[i];
  }
  if (publish<1>(acc, part, cnt, sm, &last)) {
    const double t = grid_total<1>(part, 0, sm);
    if (tid_() == 0) {
      s->pw = t;
      s->alpha = s->rro / t;
      *cnt = 0u;
    }
  }
}

// r = u0 - A u, rr = r.r; the first call of a solve fixes ||r0|| and the stop
// threshold (k_resid in 3D).
__global__ void __launch_bounds__(NT, kResident) k_resid3(Geom3 g, const double *__restrict__ Kx,
                                                         const double *__restrict__ Ky, const double *__restrict__ Kz,
                                                         const double *__restrict__ u, const double *__restrict__ u0,
                                                         double *__restrict__ r, double rx, double ry, double rz,
                                                         double eps, Scalars *s, double *part, unsigned *cnt) {
  __shared__ double sm[kWarps];
  __shared__ int last;
  double acc[1] = {0.0};
  HEAT_CELLS3(g) {
    const long long i = (long long)z * g.plane + (long long)y * g.pitch + x;
    const double rv = u0[i] - smvp3<double>(Kx, Ky, Kz, u, i, g.pitch, g.plane, rx, ry, rz);
    r[i] = rv;
    acc[0] = acc[0] + rv * rv;
  }
  if (publish<1>(acc, part, cnt, sm, &last)) {
    const double t = grid_total<1>(part, 0, sm);
    if (tid_() == 0) {
      s->rr = t;
      const double nrm = sqrt(fabs(t));
      if (s->first) {
        s->rr0 = t;
        s->stop = eps * nrm;
        s->first = 0;
      }
      s->err = nrm;
      s->done = (fabs(nrm) < s->stop) ? 1 : 0;
      *cnt = 0u;
    }
  }
}

// Mi = 1 / diag(A) on the interior.
__global__ void __launch_bounds__(NT, kResident) k_diag3(Geom3 g, const double *__restrict__ Kx,
                                                        const double *__restrict__ Ky, const double *__restrict__ Kz,
                                                        double rx, double ry, double rz, double *__restrict__ Mi) {
  HEAT_CELLS3(g) {
    const long long i = (long long)z * g.plane + (long long)y * g.pitch + x;
    Mi[i] = 1.0 / (1.0 + rz * (Kz[i + g.plane] + Kz[i]) + ry * (Ky[i + g.pitch] + Ky[i]) + rx * (Kx[i + 1] + Kx[i]));
  }
}

// FP32 copy of n consecutive FP64 values (a padded volume, halos included).
__global__ void __launch_bounds__(NT, kResident) k_flat_to_float(const double *__restrict__ a, float *__restrict__ fa,
                                                                long long n) {
  for (long long k = (long long)blockIdx.x * NT + tid_(); k < n; k += (long long)gridDim.x * NT) fa[k] = (float)a[k];
}

dim3 grid_for3(int nx, int rows) {
  int gx = (nx + BX - 1) / BX;
  if (gx > 1024) gx = 1024;
  int gy = kTargetBlocks / gx;
  const int r = (rows + BY - 1) / BY;
  if (gy > r) gy = r;
  if (gy < 1) gy = 1;
  return dim3(gx, gy);
}

void check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw Error(E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

struct Solver::Impl {
  Scalars *s64 = nullptr, *s32 = nullptr;
  double *part = nullptr;
  unsigned *cnt = nullptr;
  int *h_flag = nullptr;  // pinned, two slots
  cudaEvent_t ev[2] = {nullptr, nullptr};
  // FP32 mirror for the mixed solver
  float *f32 = nullptr;
  size_t f32_bytes = 0;
  long long pitch32 = 0;
  float *Kx = nullptr, *Ky = nullptr, *Mi = nullptr, *r = nullptr, *p = nullptr, *w = nullptr, *z = nullptr,
        *e = nullptr;
  float *Kz = nullptr;  // 3D only
  // replayed iteration chunks, rebuilt when any argument changes
  struct Chunk {
    cudaGraphExec_t exec = nullptr;
    std::string key;
  } chunk64, chunk32;

  ~Impl() {
    for (Chunk *c : {&chunk64, &chunk32})
      if (c->exec) cudaGraphExecDestroy(c->exec);
    for (cudaEvent_t x : ev)
      if (x) cudaEventDestroy(x);
    if (h_flag) cudaFreeHost(h_flag);
    cudaFree(s64);
    cudaFree(part);
    cudaFree(cnt);
    cudaFree(f32);
  }

  void ensure_base() {
    if (s64) return;
    OPSB_CUDA(cudaMalloc(&s64, 2 * sizeof(Scalars)));
    s32 = s64 + 1;
    OPSB_CUDA(cudaMalloc(&part, 2 * kMaxBlocks * sizeof(double)));
    OPSB_CUDA(cudaMalloc(&cnt, 64));
    OPSB_CUDA(cudaMemset(cnt, 0, 64));
    OPSB_CUDA(cudaMallocHost(&h_flag, 2 * sizeof(int)));
    for (cudaEvent_t &x : ev) OPSB_CUDA(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
  }

  // The 3D mixed solver's nine FP32 fields, each a padded volume of nf
  // values in the FP64 fields' flat layout, zero on every halo cell.
  void ensure_f32_flat(size_t nf, cudaStream_t st) {
    const size_t bytes = 9 * nf * sizeof(float);
    if (bytes != f32_bytes || pitch32 != -1) {
      cudaFree(f32);
      f32 = nullptr;
      OPSB_CUDA(cudaMalloc(&f32, bytes));
      f32_bytes = bytes;
      pitch32 = -1;  // the 2D layout must be rebuilt
      chunk32.key.clear();
    }
    OPSB_CUDA(cudaMemsetAsync(f32, 0, bytes, st));
    float **fields[9] = {&Kx, &Ky, &Kz, &Mi, &r, &p, &w, &z, &e};
    for (int k = 0; k < 9; k++) *fields[k] = f32 + k * nf;
  }

  // Eight FP32 fields with a one-cell ring; x = 0 of the interior starts a
  // 128-byte line.
  void ensure_f32(int nx, int ny, cudaStream_t st) {
    long long pitch = ((32 + nx + 1 + 31) / 32) * 32;
    size_t one = (size_t)pitch * (ny + 2);
    size_t bytes = 8 * one * sizeof(float);
    if (bytes != f32_bytes || pitch != pitch32) {
      cudaFree(f32);
      f32 = nullptr;
      OPSB_CUDA(cudaMalloc(&f32, bytes));
      f32_bytes = bytes;
      pitch32 = pitch;
      chunk32.key.clear();
    }
    OPSB_CUDA(cudaMemsetAsync(f32, 0, bytes, st));
    float **fields[8] = {&Kx, &Ky, &Mi, &r, &p, &w, &z, &e};
    for (int k = 0; k < 8; k++) *fields[k] = f32 + k * one + pitch + 32;
  }
};

Solver::Solver() : m_(new Impl) {}
Solver::~Solver() { delete m_; }

namespace {

dim3 grid_for(int nx, int ny) {
  int gx = (nx + BX - 1) / BX;
  if (gx > 1024) gx = 1024;
  int gy = kTargetBlocks / gx;
  const int rows = (ny + BY - 1) / BY;
  if (gy > rows) gy = rows;
  if (gy < 1) gy = 1;
  return dim3(gx, gy);
}

std::string key_of(std::initializer_list<const void *> ptrs, std::initializer_list<double> vals) {
  std::string k;
  for (const void *p : ptrs) k.append(reinterpret_cast<const char *>(&p), sizeof(p));
  for (double v : vals) k.append(reinterpret_cast<const char *>(&v), sizeof(v));
  return k;
}

// Launches chunks of iterations until the solver flag says done; the host
// reads the flag of chunk c while chunk c+1 runs.
long long run_chunks(cudaGraphExec_t g, const Scalars *s, int max_iters, int *h_flag, cudaEvent_t *ev,
                     cudaStream_t st, int launches_per_chunk) {
  long long launches = 0;
  const int max_chunks = max_iters / kChunk + 2;
  for (int c = 0; c < max_chunks; c++) {
    OPSB_CUDA(cudaGraphLaunch(g, st));
    launches += launches_per_chunk;
    OPSB_CUDA(cudaMemcpyAsync(&h_flag[c & 1], &s->done, sizeof(int), cudaMemcpyDeviceToHost, st));
    OPSB_CUDA(cudaEventRecord(ev[c & 1], st));
    if (c > 0) {
      OPSB_CUDA(cudaEventSynchronize(ev[(c - 1) & 1]));
      if (h_flag[(c - 1) & 1]) break;
    }
  }
  OPSB_CUDA(cudaStreamSynchronize(st));
  return launches;
}

template <class F>
cudaGraphExec_t capture(cudaStream_t st, F body) {
  cudaGraph_t graph = nullptr;
  OPSB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  body();
  cudaError_t le = cudaGetLastError();
  OPSB_CUDA(cudaStreamEndCapture(st, &graph));
  if (le != cudaSuccess) {
    cudaGraphDestroy(graph);
    throw Error(E_CUDA, std::string("heat solver capture: ") + cudaGetErrorString(le));
  }
  cudaGraphExec_t exec = nullptr;
  cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  OPSB_CUDA(ie);
  return exec;
}

void validate(const Field2D &f) {
  if (f.nx < 1 || f.ny < 1) throw Error(E_ARG, "heat solver: empty interior");
  if (f.pitch < f.nx + 2) throw Error(E_ARG, "heat solver: pitch smaller than the row");
  if (!f.Kx || !f.Ky || !f.u0 || !f.u || !f.r || !f.w || !f.p || !f.z || !f.Mi)
    throw Error(E_ARG, "heat solver: null field");
  if ((long long)f.ny * f.pitch > (1LL << 40)) throw Error(E_ARG, "heat solver: field too large");
}

Scalars fresh(double stop) {
  Scalars h;
  memset(&h, 0, sizeof(h));
  h.first = 1;
  h.stop = stop;
  return h;
}

}  // namespace

void Solver::pcg_fp64(const Field2D &f, double rx, double ry, bool precond, bool true_stop, double eps,
                      int max_iters, cudaStream_t st, SolveStats *out) {
  validate(f);
  Impl &m = *m_;
  m.ensure_base();
  launches_ = 0;
  const Geom g{f.nx, f.ny, f.pitch};
  const dim3 grid = grid_for(f.nx, f.ny), block(BX, BY);
  Scalars h = fresh(0.0);
  OPSB_CUDA(cudaMemcpyAsync(m.s64, &h, sizeof(h), cudaMemcpyHostToDevice, st));
  // initial residual (tea_solve.cpp:105-114) and cg_init
  k_resid<<<grid, block, 0, st>>>(g, f.Kx, f.Ky, f.u, f.u0, f.r, rx, ry, eps, m.s64, m.part, m.cnt);
  if (precond)
    k_init<true><<<grid, block, 0, st>>>(g, f.r, f.Mi, f.z, f.p, max_iters, m.s64, m.part, m.cnt);
  else
    k_init<false><<<grid, block, 0, st>>>(g, f.r, f.Mi, f.z, f.p, max_iters, m.s64, m.part, m.cnt);
  check_launch("heat solver init");
  launches_ += 2;
  if (max_iters > 0) {
    const std::string key = key_of({f.Kx, f.Ky, f.u, f.r, f.w, f.p, f.z, f.Mi},
                                   {rx, ry, (double)f.nx, (double)f.ny, (double)f.pitch, precond ? 1.0 : 0.0,
                                    true_stop ? 1.0 : 0.0});
    if (m.chunk64.key != key) {
      if (m.chunk64.exec) cudaGraphExecDestroy(m.chunk64.exec);
      m.chunk64.exec = nullptr;
      m.chunk64.key.clear();
      double *zsrc = precond ? f.z : f.r;
      m.chunk64.exec = capture(st, [&] {
        for (int it = 0; it < kChunk; it++) {
          k_w<double><<<grid, block, 0, st>>>(g, f.Kx, f.Ky, f.p, f.w, rx, ry, m.s64, m.part, m.cnt);
          if (precond && true_stop)
            k_ur<double, true, STOP_TRUE><<<grid, block, 0, st>>>(g, f.u, f.p, f.r, f.w, f.Mi, f.z, m.s64, m.part,
                                                                  m.cnt);
          else if (precond)
            k_ur<double, true, STOP_TEALEAF><<<grid, block, 0, st>>>(g, f.u, f.p, f.r, f.w, f.Mi, f.z, m.s64,
                                                                     m.part, m.cnt);
          else
            k_ur<double, false, STOP_TEALEAF><<<grid, block, 0, st>>>(g, f.u, f.p, f.r, f.w, f.Mi, f.z, m.s64,
                                                                      m.part, m.cnt);
          k_p<double><<<grid, block, 0, st>>>(g, f.p, zsrc, m.s64);
        }
      });
      m.chunk64.key = key;
    }
    launches_ += run_chunks(m.chunk64.exec, m.s64, max_iters, m.h_flag, m.ev, st, 3 * kChunk);
  }
  OPSB_CUDA(cudaMemcpyAsync(&h, m.s64, sizeof(h), cudaMemcpyDeviceToHost, st));
  OPSB_CUDA(cudaStreamSynchronize(st));
  const double r0 = sqrt(fabs(h.rr0));
  out->initial_residual = r0;
  out->error = h.err;
  out->converged = h.done == 1 || (max_iters <= 0 && h.err < h.stop);
  // the reference reports n - 1: one less than the iteration that met the test
  out->iterations = h.done == 1 ? h.iters - 1 : h.iters;
  out->outer = 0;
  // true FP64 residual at exit, computed into w (which the next solve
  // overwrites before reading), so r keeps the loop's recursive residual.
  Scalars t = fresh(0.0);
  OPSB_CUDA(cudaMemcpyAsync(m.s32, &t, sizeof(t), cudaMemcpyHostToDevice, st));
  k_resid<<<grid, block, 0, st>>>(g, f.Kx, f.Ky, f.u, f.u0, f.w, rx, ry, 0.0, m.s32, m.part, m.cnt);
  check_launch("heat solver residual");
  launches_ += 1;
  OPSB_CUDA(cudaMemcpyAsync(&t, m.s32, sizeof(t), cudaMemcpyDeviceToHost, st));
  OPSB_CUDA(cudaStreamSynchronize(st));
  out->true_residual = sqrt(fabs(t.rr));
}

void Solver::pcg_mixed(const Field2D &f, double rx, double ry, bool precond, double eps, double delta,
                       int max_iters, cudaStream_t st, SolveStats *out) {
  validate(f);
  if (!(delta > 0.0 && delta < 1.0)) throw Error(E_ARG, "heat solver: reliable-update delta must be in (0, 1)");
  Impl &m = *m_;
  m.ensure_base();
  m.ensure_f32(f.nx, f.ny, st);
  launches_ = 0;
  const Geom g{f.nx, f.ny, f.pitch}, g32{f.nx, f.ny, m.pitch32};
  const dim3 grid = grid_for(f.nx, f.ny), block(BX, BY);
  const float rxf = (float)rx, ryf = (float)ry;
  k_to_float<<<grid_for(f.nx + 2, f.ny + 2), block, 0, st>>>(g, g32, f.Kx, f.Ky, precond ? f.Mi : nullptr, m.Kx,
                                                              m.Ky, m.Mi);
  Scalars h = fresh(0.0);
  OPSB_CUDA(cudaMemcpyAsync(m.s64, &h, sizeof(h), cudaMemcpyHostToDevice, st));
  k_resid<<<grid, block, 0, st>>>(g, f.Kx, f.Ky, f.u, f.u0, f.r, rx, ry, eps, m.s64, m.part, m.cnt);
  check_launch("heat solver init");
  launches_ += 2;
  OPSB_CUDA(cudaMemcpyAsync(&h, m.s64, sizeof(h), cudaMemcpyDeviceToHost, st));
  OPSB_CUDA(cudaStreamSynchronize(st));
  const double r0 = sqrt(fabs(h.rr0));
  out->initial_residual = r0;
  const std::string key = key_of({m.Kx, m.Ky, m.e, m.r, m.w, m.p, m.z, m.Mi},
                                 {(double)rxf, (double)ryf, (double)f.nx, (double)f.ny, (double)m.pitch32,
                                  precond ? 1.0 : 0.0});
  if (m.chunk32.key != key) {
    if (m.chunk32.exec) cudaGraphExecDestroy(m.chunk32.exec);
    m.chunk32.exec = nullptr;
    m.chunk32.key.clear();
    float *zsrc = precond ? m.z : m.r;
    m.chunk32.exec = capture(st, [&] {
      for (int it = 0; it < kChunk; it++) {
        k_w<float><<<grid, block, 0, st>>>(g32, m.Kx, m.Ky, m.p, m.w, rxf, ryf, m.s32, m.part, m.cnt);
        if (precond)
          k_ur<float, true, STOP_RELIABLE><<<grid, block, 0, st>>>(g32, m.e, m.p, m.r, m.w, m.Mi, m.z, m.s32,
                                                                   m.part, m.cnt);
        else
          k_ur<float, false, STOP_RELIABLE><<<grid, block, 0, st>>>(g32, m.e, m.p, m.r, m.w, m.Mi, m.z, m.s32,
                                                                    m.part, m.cnt);
        k_p<float><<<grid, block, 0, st>>>(g32, m.p, zsrc, m.s32);
      }
    });
    m.chunk32.key = key;
  }
  float *zsrc = precond ? m.z : m.r;
  int updates = 0, iters = 0;
  double scale = 1.0;
  bool done = h.done == 1 || r0 == 0.0;
  Scalars in;
  memset(&in, 0, sizeof(in));
  while (!done) {
    if (precond)
      k_reinit32<true><<<grid, block, 0, st>>>(g, g32, f.r, m.r, m.Mi, m.z, updates == 0, eps, scale, delta,
                                               max_iters, m.s32, m.part, m.cnt);
    else
      k_reinit32<false><<<grid, block, 0, st>>>(g, g32, f.r, m.r, m.Mi, m.z, updates == 0, eps, scale, delta,
                                                max_iters, m.s32, m.part, m.cnt);
    k_p<float><<<grid, block, 0, st>>>(g32, m.p, zsrc, m.s32);
    check_launch("heat solver reliable update");
    launches_ += 2;
    launches_ += run_chunks(m.chunk32.exec, m.s32, max_iters, m.h_flag, m.ev, st, 3 * kChunk);
    OPSB_CUDA(cudaMemcpyAsync(&in, m.s32, sizeof(in), cudaMemcpyDeviceToHost, st));
    k_update<<<grid, block, 0, st>>>(g, g32, f.u, m.e);
    k_resid<<<grid, block, 0, st>>>(g, f.Kx, f.Ky, f.u, f.u0, f.r, rx, ry, eps, m.s64, m.part, m.cnt);
    check_launch("heat solver reliable update");
    launches_ += 2;
    OPSB_CUDA(cudaMemcpyAsync(&h, m.s64, sizeof(h), cudaMemcpyDeviceToHost, st));
    OPSB_CUDA(cudaStreamSynchronize(st));
    updates++;
    iters = in.iters;
    done = h.done == 1;
    if (done || in.done == 2 || in.iters >= max_iters || updates > 10000) break;
    // the estimate said converged but the FP64 residual disagrees: tighten it
    if (in.done == 1) scale *= 0.1;
  }
  out->iterations = iters;
  out->outer = updates;
  out->converged = done;
  out->error = h.err;
  out->true_residual = h.err;
}


namespace {
void validate3(const Field3D &f) {
  if (f.nx < 1 || f.ny < 1 || f.nz < 1) throw Error(E_ARG, "heat solver 3D: empty interior");
  if (f.pitch < f.nx + 2 || f.plane != f.pitch * (f.ny + 2))
    throw Error(E_ARG, "heat solver 3D: pitch >= nx + 2 and plane == pitch * (ny + 2) required");
  if (!f.Kx || !f.Ky || !f.Kz || !f.u0 || !f.u || !f.r || !f.w || !f.p || !f.z || !f.Mi)
    throw Error(E_ARG, "heat solver 3D: null field");
  if ((long long)(f.ny + 2) * (f.nz + 2) > (1LL << 30) || f.plane * (f.nz + 2) > (1LL << 40))
    throw Error(E_ARG, "heat solver 3D: field too large");
}
}  // namespace

void Solver::diag3(const Field3D &f, double rx, double ry, double rz, cudaStream_t st) {
  validate3(f);
  k_diag3<<<grid_for3(f.nx, f.ny * f.nz), dim3(BX, BY), 0, st>>>(Geom3{f.nx, f.ny, f.nz, f.pitch, f.plane}, f.Kx,
                                                                   f.Ky, f.Kz, rx, ry, rz, f.Mi);
  check_launch("heat solver 3D diagonal");
}

void Solver::pcg3d(const Field3D &f, double rx, double ry, double rz, bool true_stop, double eps, int max_iters,
                   cudaStream_t st, SolveStats *out) {
  validate3(f);
  Impl &m = *m_;
  m.ensure_base();
  launches_ = 0;
  const Geom3 g{f.nx, f.ny, f.nz, f.pitch, f.plane};
  const dim3 grid3 = grid_for3(f.nx, f.ny * f.nz), block(BX, BY);
  // the pointwise kernels see the padded volume as rows of `pitch`
  const long long off = f.plane + f.pitch + 1;
  const int rows = (f.ny + 2) * (f.nz + 2);
  const Geom gf{(int)f.pitch, rows, f.pitch};
  const dim3 gridf = grid_for((int)f.pitch, rows);
  double *u = f.u - off, *r = f.r - off, *w = f.w - off, *p = f.p - off, *z = f.z - off;
  const double *Mi = f.Mi - off;
  Scalars h = fresh(0.0);
  OPSB_CUDA(cudaMemcpyAsync(m.s64, &h, sizeof(h), cudaMemcpyHostToDevice, st));
  k_resid3<<<grid3, block, 0, st>>>(g, f.Kx, f.Ky, f.Kz, f.u, f.u0, f.r, rx, ry, rz, eps, m.s64, m.part, m.cnt);
  k_init<true><<<gridf, block, 0, st>>>(gf, r, Mi, z, p, max_iters, m.s64, m.part, m.cnt);
  check_launch("heat solver 3D init");
  launches_ += 2;
  if (max_iters > 0) {
    const std::string key = "3d" + key_of({f.Kx, f.Ky, f.Kz, f.u, f.r, f.w, f.p, f.z, f.Mi},
                                          {rx, ry, rz, (double)f.nx, (double)f.ny, (double)f.nz, (double)f.pitch,
                                           true_stop ? 1.0 : 0.0});
    if (m.chunk64.key != key) {
      if (m.chunk64.exec) cudaGraphExecDestroy(m.chunk64.exec);
      m.chunk64.exec = nullptr;
      m.chunk64.key.clear();
      m.chunk64.exec = capture(st, [&] {
        for (int it = 0; it < kChunk; it++) {
          k_w3<double><<<grid3, block, 0, st>>>(g, f.Kx, f.Ky, f.Kz, f.p, f.w, rx, ry, rz, m.s64, m.part, m.cnt);
          if (true_stop)
            k_ur<double, true, STOP_TRUE><<<gridf, block, 0, st>>>(gf, u, p, r, w, Mi, z, m.s64, m.part, m.cnt);
          else
            k_ur<double, true, STOP_TEALEAF><<<gridf, block, 0, st>>>(gf, u, p, r, w, Mi, z, m.s64, m.part, m.cnt);
          k_p<double><<<gridf, block, 0, st>>>(gf, p, z, m.s64);
        }
      });
      m.chunk64.key = key;
    }
    launches_ += run_chunks(m.chunk64.exec, m.s64, max_iters, m.h_flag, m.ev, st, 3 * kChunk);
  }
  OPSB_CUDA(cudaMemcpyAsync(&h, m.s64, sizeof(h), cudaMemcpyDeviceToHost, st));
  OPSB_CUDA(cudaStreamSynchronize(st));
  out->initial_residual = sqrt(fabs(h.rr0));
  out->error = h.err;
  out->converged = h.done == 1 || (max_iters <= 0 && h.err < h.stop);
  out->iterations = h.done == 1 ? h.iters - 1 : h.iters;
  out->outer = 0;
  Scalars t = fresh(0.0);
  OPSB_CUDA(cudaMemcpyAsync(m.s32, &t, sizeof(t), cudaMemcpyHostToDevice, st));
  k_resid3<<<grid3, block, 0, st>>>(g, f.Kx, f.Ky, f.Kz, f.u, f.u0, f.w, rx, ry, rz, 0.0, m.s32, m.part, m.cnt);
  check_launch("heat solver 3D residual");
  launches_ += 1;
  OPSB_CUDA(cudaMemcpyAsync(&t, m.s32, sizeof(t), cudaMemcpyDeviceToHost, st));
  OPSB_CUDA(cudaStreamSynchronize(st));
  out->true_residual = sqrt(fabs(t.rr));
}

void Solver::pcg3d_mixed(const Field3D &f, double rx, double ry, double rz, double eps, double delta, int max_iters,
                         cudaStream_t st, SolveStats *out) {
  validate3(f);
  if (!(delta > 0.0 && delta < 1.0)) throw Error(E_ARG, "heat solver: reliable-update delta must be in (0, 1)");
  Impl &m = *m_;
  m.ensure_base();
  const long long off = f.plane + f.pitch + 1;
  const size_t nf = (size_t)f.plane * (f.nz + 2);
  m.ensure_f32_flat(nf, st);
  launches_ = 0;
  const Geom3 g{f.nx, f.ny, f.nz, f.pitch, f.plane};
  const dim3 grid3 = grid_for3(f.nx, f.ny * f.nz), block(BX, BY);
  const int rows = (f.ny + 2) * (f.nz + 2);
  const Geom gf{(int)f.pitch, rows, f.pitch};
  const dim3 gridf = grid_for((int)f.pitch, rows);
  const dim3 grid1((unsigned)std::min<long long>(((long long)nf + NT - 1) / NT, 148LL * 16));
  const float rxf = (float)rx, ryf = (float)ry, rzf = (float)rz;
  k_flat_to_float<<<grid1, block, 0, st>>>(f.Kx - off, m.Kx, (long long)nf);
  k_flat_to_float<<<grid1, block, 0, st>>>(f.Ky - off, m.Ky, (long long)nf);
  k_flat_to_float<<<grid1, block, 0, st>>>(f.Kz - off, m.Kz, (long long)nf);
  k_flat_to_float<<<grid1, block, 0, st>>>(f.Mi - off, m.Mi, (long long)nf);
  Scalars h = fresh(0.0);
  OPSB_CUDA(cudaMemcpyAsync(m.s64, &h, sizeof(h), cudaMemcpyHostToDevice, st));
  k_resid3<<<grid3, block, 0, st>>>(g, f.Kx, f.Ky, f.Kz, f.u, f.u0, f.r, rx, ry, rz, eps, m.s64, m.part, m.cnt);
  check_launch("heat solver 3D init");
  launches_ += 5;
  OPSB_CUDA(cudaMemcpyAsync(&h, m.s64, sizeof(h), cudaMemcpyDeviceToHost, st));
  OPSB_CUDA(cudaStreamSynchronize(st));
  const double r0 = sqrt(fabs(h.rr0));
  out->initial_residual = r0;
  const std::string key = "3d" + key_of({m.Kx, m.Ky, m.Kz, m.e, m.r, m.w, m.p, m.z, m.Mi},
                                        {(double)rxf, (double)ryf, (double)rzf, (double)f.nx, (double)f.ny,
                                         (double)f.nz, (double)f.pitch});
  if (m.chunk32.key != key) {
    if (m.chunk32.exec) cudaGraphExecDestroy(m.chunk32.exec);
    m.chunk32.exec = nullptr;
    m.chunk32.key.clear();
    m.chunk32.exec = capture(st, [&] {
      for (int it = 0; it < kChunk; it++) {
        k_w3<float><<<grid3, block, 0, st>>>(g, m.Kx + off, m.Ky + off, m.Kz + off, m.p + off, m.w + off, rxf, ryf,
                                             rzf, m.s32, m.part, m.cnt);
        k_ur<float, true, STOP_RELIABLE><<<gridf, block, 0, st>>>(gf, m.e, m.p, m.r, m.w, m.Mi, m.z, m.s32, m.part,
                                                                  m.cnt);
        k_p<float><<<gridf, block, 0, st>>>(gf, m.p, m.z, m.s32);
      }
    });
    m.chunk32.key = key;
  }
  int updates = 0, iters = 0;
  double scale = 1.0;
  bool done = h.done == 1 || r0 == 0.0;
  Scalars in;
  memset(&in, 0, sizeof(in));
  while (!done) {
    k_reinit32<true><<<gridf, block, 0, st>>>(gf, gf, f.r - off, m.r, m.Mi, m.z, updates == 0, eps, scale, delta,
                                              max_iters, m.s32, m.part, m.cnt);
    k_p<float><<<gridf, block, 0, st>>>(gf, m.p, m.z, m.s32);
    check_launch("heat solver 3D reliable update");
    launches_ += 2;
    launches_ += run_chunks(m.chunk32.exec, m.s32, max_iters, m.h_flag, m.ev, st, 3 * kChunk);
    OPSB_CUDA(cudaMemcpyAsync(&in, m.s32, sizeof(in), cudaMemcpyDeviceToHost, st));
    k_update<<<gridf, block, 0, st>>>(gf, gf, f.u - off, m.e);
    k_resid3<<<grid3, block, 0, st>>>(g, f.Kx, f.Ky, f.Kz, f.u, f.u0, f.r, rx, ry, rz, eps, m.s64, m.part, m.cnt);
    check_launch("heat solver 3D reliable update");
    launches_ += 2;
    OPSB_CUDA(cudaMemcpyAsync(&h, m.s64, sizeof(h), cudaMemcpyDeviceToHost, st));
    OPSB_CUDA(cudaStreamSynchronize(st));
    updates++;
    iters = in.iters;
    done = h.done == 1;
    if (done || in.done == 2 || in.iters >= max_iters || updates > 10000) break;
    if (in.done == 1) scale *= 0.1;  // the estimate said converged, the FP64 residual disagrees
  }
  out->iterations = iters;
  out->outer = updates;
  out->converged = done;
  out->error = h.err;
  out->true_residual = h.err;
}

void Solver::diag(const Field2D &f, double rx, double ry, cudaStream_t st) {
  validate(f);
  k_diag<<<grid_for(f.nx, f.ny), dim3(BX, BY), 0, st>>>(Geom{f.nx, f.ny, f.pitch}, f.Kx, f.Ky, rx, ry, f.Mi);
  check_launch("heat solver diagonal");
}

double Solver::residual(const Field2D &f, double rx, double ry, double *outp, cudaStream_t st) {
  validate(f);
  Impl &m = *m_;
  m.ensure_base();
  Scalars t = fresh(0.0);
  OPSB_CUDA(cudaMemcpyAsync(m.s32, &t, sizeof(t), cudaMemcpyHostToDevice, st));
  k_resid<<<grid_for(f.nx, f.ny), dim3(BX, BY), 0, st>>>(Geom{f.nx, f.ny, f.pitch}, f.Kx, f.Ky, f.u, f.u0, outp, rx,
                                                         ry, 0.0, m.s32, m.part, m.cnt);
  check_launch("heat residual");
  OPSB_CUDA(cudaMemcpyAsync(&t, m.s32, sizeof(t), cudaMemcpyDeviceToHost, st));
  OPSB_CUDA(cudaStreamSynchronize(st));
  return sqrt(fabs(t.rr));
}

void Solver::fcg(const Field2D &f, double rx, double ry, double eps, int max_iters, const Precond &M, int window,
                 cudaStream_t st, SolveStats *out, const Precond *fallback, bool chunked) {
  validate(f);
  Impl &m = *m_;
  m.ensure_base();
  launches_ = 0;
  const Geom g{f.nx, f.ny, f.pitch};
  const dim3 grid = grid_for(f.nx, f.ny), block(BX, BY);
  Scalars h = fresh(0.0);
  h.max_iters = max_iters;
  OPSB_CUDA(cudaMemcpyAsync(m.s64, &h, sizeof(h), cudaMemcpyHostToDevice, st));
  k_resid<<<grid, block, 0, st>>>(g, f.Kx, f.Ky, f.u, f.u0, f.r, rx, ry, eps, m.s64, m.part, m.cnt);
  check_launch("fcg init");
  launches_ += 1;
  bool learned = static_cast<bool>(M);
  auto precond = [&] {
    if (learned) {
      launches_ += M(f.r, f.z, st);
    } else if (fallback && *fallback) {
      launches_ += (*fallback)(f.r, f.z, st);
    } else {
      k_jacobi<<<grid, block, 0, st>>>(g, f.Mi, f.r, f.z);
      launches_ += 1;
    }
  };
  OPSB_CUDA(cudaMemcpyAsync(&h, m.s64, sizeof(h), cudaMemcpyDeviceToHost, st));
  OPSB_CUDA(cudaStreamSynchronize(st));
  const double r0 = sqrt(fabs(h.rr0));
  out->initial_residual = r0;
  out->fallbacks = 0;
  bool done = h.done == 1 || r0 == 0.0;
  if (!done) {
    // the initial residual kernel leaves done = 0 and iters = 0
    precond();
    k_fp<<<grid, block, 0, st>>>(g, f.p, f.z, m.s64, 1);
    launches_ += 1;
  }
  bool host_loop = true;
  if (chunked && window < 64 && !done) {
    host_loop = false;
    // Replayed chunks of kFcgChunk iterations (w = A p, update, precondition,
    // beta, direction); the device stops them (done != 0) and the host reads
    // the flag one chunk behind. A restart (done 4 or 5) falls back to the
    // Jacobi (or fallback) preconditioner and continues with that chunk.
    // The graphs hold this call's pointers and are rebuilt per call.
    constexpr int kFcgChunk = 4;
    int set[2] = {learned ? window : 0, 0};
    OPSB_CUDA(cudaMemcpyAsync(&m.s64->window, set, sizeof(set), cudaMemcpyHostToDevice, st));
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};  // learned, fallback
    long long per_chunk[2] = {0, 0};
    try {
      while (!done) {
        const int which = learned ? 0 : 1;
        if (!graphs[which]) {
          const long long before = launches_;
          graphs[which] = capture(st, [&] {
            for (int it = 0; it < kFcgChunk; it++) {
              k_fw<<<grid, block, 0, st>>>(g, f.Kx, f.Ky, f.p, f.r, f.w, rx, ry, m.s64, m.part, m.cnt);
              k_fupd<<<grid, block, 0, st>>>(g, f.u, f.p, f.r, f.w, m.s64, m.part, m.cnt);
              launches_ += 2;
              precond();
              k_fzw<<<grid, block, 0, st>>>(g, f.z, f.w, m.s64, m.part, m.cnt);
              k_fp<<<grid, block, 0, st>>>(g, f.p, f.z, m.s64, 0);
              launches_ += 2;
            }
          });
          per_chunk[which] = launches_ - before;
          launches_ = before;
        }
        // run_chunks stops after (its bound) / kChunk + 2 chunks at most; the
        // device stops them first (done 2 at max_iters)
        launches_ += run_chunks(graphs[which], m.s64, (max_iters / kFcgChunk + 2) * kChunk, m.h_flag, m.ev, st,
                                per_chunk[which]);
        OPSB_CUDA(cudaMemcpyAsync(&h, m.s64, sizeof(h), cudaMemcpyDeviceToHost, st));
        OPSB_CUDA(cudaStreamSynchronize(st));
        if (h.done == 1 || h.done == 2 || h.done == 0) break;
        // done 4 (lost curvature) or 5 (not halved over the window): restart
        if (learned) out->fallbacks++;
        learned = false;
        const int zero3[3] = {0, 0, 0};  // done = 0; window = hcount = 0 (no restart test on the fallback)
        OPSB_CUDA(cudaMemcpyAsync(&m.s64->done, zero3, sizeof(int), cudaMemcpyHostToDevice, st));
        OPSB_CUDA(cudaMemcpyAsync(&m.s64->window, zero3 + 1, 2 * sizeof(int), cudaMemcpyHostToDevice, st));
        precond();
        k_fp<<<grid, block, 0, st>>>(g, f.p, f.z, m.s64, 1);
        launches_ += 1;
      }
    } catch (...) {
      for (cudaGraphExec_t x : graphs)
        if (x) cudaGraphExecDestroy(x);
      throw;
    }
    for (cudaGraphExec_t x : graphs)
      if (x) cudaGraphExecDestroy(x);
  }
  std::vector<double> hist;
  while (!done && host_loop) {
    k_fw<<<grid, block, 0, st>>>(g, f.Kx, f.Ky, f.p, f.r, f.w, rx, ry, m.s64, m.part, m.cnt);
    k_fupd<<<grid, block, 0, st>>>(g, f.u, f.p, f.r, f.w, m.s64, m.part, m.cnt);
    check_launch("fcg iteration");
    launches_ += 2;
    OPSB_CUDA(cudaMemcpyAsync(&h, m.s64, sizeof(h), cudaMemcpyDeviceToHost, st));
    OPSB_CUDA(cudaStreamSynchronize(st));
    if (h.done == 1 || h.done == 2) break;
    bool restart = false;
    if (h.done == 4) {
      restart = true;  // lost positive curvature: fall back to Jacobi and restart the recursion
    } else {
      hist.push_back(h.err);
      const size_t k = hist.size();
      if (learned && window > 0 && k > (size_t)window && hist[k - 1] > 0.5 * hist[k - 1 - window]) restart = true;
    }
    if (restart) {
      if (learned) out->fallbacks++;
      learned = false;
      hist.clear();
      int zero = 0;
      OPSB_CUDA(cudaMemcpyAsync(&m.s64->done, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
      precond();
      k_fp<<<grid, block, 0, st>>>(g, f.p, f.z, m.s64, 1);
      launches_ += 1;
      continue;
    }
    precond();
    k_fzw<<<grid, block, 0, st>>>(g, f.z, f.w, m.s64, m.part, m.cnt);
    k_fp<<<grid, block, 0, st>>>(g, f.p, f.z, m.s64, 0);
    check_launch("fcg direction");
    launches_ += 2;
  }
  out->iterations = h.iters;
  out->converged = h.done == 1 || done;
  out->error = h.err;
  out->outer = 0;
  // true FP64 residual at exit (into w)
  Scalars t = fresh(0.0);
  OPSB_CUDA(cudaMemcpyAsync(m.s32, &t, sizeof(t), cudaMemcpyHostToDevice, st));
  k_resid<<<grid, block, 0, st>>>(g, f.Kx, f.Ky, f.u, f.u0, f.w, rx, ry, 0.0, m.s32, m.part, m.cnt);
  check_launch("fcg residual");
  launches_ += 1;
  OPSB_CUDA(cudaMemcpyAsync(&t, m.s32, sizeof(t), cudaMemcpyDeviceToHost, st));
  OPSB_CUDA(cudaStreamSynchronize(st));
  out->true_residual = sqrt(fabs(t.rr));
}

}  // namespace heat
}  // namespace opsb
