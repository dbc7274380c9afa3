// Aggregation multigrid V-cycle for the TeaLeaf 2D heat operator; the
// hierarchy and the cycle are described in heat_mg.h.
//
// Storage: every level keeps its FP32 arrays without a halo ring, rows of
// `pitch` elements (a multiple of 32, at least nx + 1 so that a row holds all
// nx + 1 x-faces); the y-face array has ny + 1 rows. Face x of a row is the
// face between cells x - 1 and x, so cell x reads faces x and x + 1 of its
// row and y-faces from its own row and the next. Neighbours outside the
// domain hold zero, so their terms are dropped while their face weights stay
// in the diagonal (as the halo of the FP64 operator does).
//
// Every kernel is a streaming pass over one level (HBM-bound on the fine
// levels): the fine level of one cycle costs five passes (first pre-sweep
// with the FP64 -> FP32 copy of r, second pre-sweep, residual + restriction,
// prolongation fused into the first post-sweep, last post-sweep writing the
// FP64 result), about 106 bytes per fine cell; the coarser levels add a third.
#include <algorithm>
#include <string>

#include "heat_mg.h"
#include "runtime.h"

namespace opsb {
namespace heat {

namespace {

constexpr int BX = 128, BY = 2;
constexpr int kCoarseThreads = Multigrid::kCoarsest * Multigrid::kCoarsest;

struct LV {
  int nx, ny;
  long long P;
  const float *m, *ax, *ay;
};

void check(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw Error(E_CUDA, std::string("multigrid ") + what + ": " + cudaGetErrorString(e));
}

dim3 grid_of(int nx, int ny) {
  const int gx = (nx + BX - 1) / BX;
  const int gy = std::min((ny + BY - 1) / BY, 32768);
  return dim3(gx, gy);
}

#define MG_CELLS(L)                                                                   \
  for (int y = blockIdx.y * BY + threadIdx.y; y < (L).ny; y += gridDim.y * BY)        \
    for (int x = blockIdx.x * BX + threadIdx.x; x < (L).nx; x += gridDim.x * BX)

// Diagonal of cell i: its mass plus its four face weights.
template <bool UNIT>
__device__ __forceinline__ float diag(const LV &L, long long i, float aw, float ae, float as, float an) {
  return (UNIT ? 1.0f : L.m[i]) + aw + ae + as + an;
}

// r - A z at (x, y), with z read through `zf(x, y)`; also returns the diagonal.
template <bool UNIT, class ZF>
__device__ __forceinline__ float resid(const LV &L, int x, int y, float rv, const ZF &zf, float &c) {
  const long long i = (long long)y * L.P + x;
  const float aw = L.ax[i], ae = L.ax[i + 1], as = L.ay[i], an = L.ay[i + L.P];
  c = diag<UNIT>(L, i, aw, ae, as, an);
  float s = rv - c * zf(x, y);
  if (x > 0) s += aw * zf(x - 1, y);
  if (x < L.nx - 1) s += ae * zf(x + 1, y);
  if (y > 0) s += as * zf(x, y - 1);
  if (y < L.ny - 1) s += an * zf(x, y + 1);
  return s;
}

// First pre-sweep from z = 0: z = omega r / c. On level 0 (R64) r arrives in
// FP64 with the fields' pitch `fp` and its FP32 copy is kept in `r32`.
template <bool UNIT, bool R64>
__global__ void __launch_bounds__(BX *BY) k_pre_first(LV L, const double *__restrict__ r64, long long fp,
                                                      float *__restrict__ r32, float *__restrict__ zout,
                                                      float omega) {
  MG_CELLS(L) {
    const long long i = (long long)y * L.P + x;
    float rv;
    if (R64) {
      rv = (float)r64[(long long)y * fp + x];
      r32[i] = rv;
    } else {
      rv = r32[i];
    }
    const float c = diag<UNIT>(L, i, L.ax[i], L.ax[i + 1], L.ay[i], L.ay[i + L.P]);
    zout[i] = omega * rv / c;
  }
}

// zout = zin + omega (r - A zin) / c; with OUT64 the result goes to the FP64
// field z64 (pitch fp) instead.
template <bool UNIT, bool OUT64>
__global__ void __launch_bounds__(BX *BY) k_smooth(LV L, const float *__restrict__ r, const float *__restrict__ zin,
                                                   float *__restrict__ zout, double *__restrict__ z64, long long fp,
                                                   float omega) {
  auto zf = [&](int xx, int yy) { return zin[(long long)yy * L.P + xx]; };
  MG_CELLS(L) {
    const long long i = (long long)y * L.P + x;
    float c;
    const float s = resid<UNIT>(L, x, y, r[i], zf, c);
    const float v = zin[i] + omega * s / c;
    if (OUT64) z64[(long long)y * fp + x] = (double)v;
    else zout[i] = v;
  }
}

// First post-sweep with the coarse correction folded in: z' = zin + P e
// (each cell takes its aggregate's value of e), then one damped-Jacobi sweep
// on z'.
template <bool UNIT, bool OUT64>
__global__ void __launch_bounds__(BX *BY) k_post_first(LV L, const float *__restrict__ r, const float *__restrict__ zin,
                                                       const float *__restrict__ e, long long eP,
                                                       float *__restrict__ zout, double *__restrict__ z64,
                                                       long long fp, float omega) {
  MG_CELLS(L) {
    const long long i = (long long)y * L.P + x;
    // the cell's aggregate value and, across the aggregate's edge on each
    // axis, the neighbouring aggregate's (the other side shares the cell's)
    const float *ec = e + (long long)(y >> 1) * eP + (x >> 1);
    const float e0 = ec[0];
    const float ew = (x & 1) ? e0 : (x > 0 ? ec[-1] : 0.f);
    const float ee = (x & 1) ? (x < L.nx - 1 ? ec[1] : 0.f) : e0;
    const float es = (y & 1) ? e0 : (y > 0 ? ec[-eP] : 0.f);
    const float en = (y & 1) ? (y < L.ny - 1 ? ec[eP] : 0.f) : e0;
    auto zf = [&](int xx, int yy) {
      const float zv = zin[(long long)yy * L.P + xx];
      return zv + (xx < x ? ew : xx > x ? ee : yy < y ? es : yy > y ? en : e0);
    };
    float c;
    const float s = resid<UNIT>(L, x, y, r[i], zf, c);
    const float v = zf(x, y) + omega * s / c;
    if (OUT64) z64[(long long)y * fp + x] = (double)v;
    else zout[i] = v;
  }
}

// Coarse right-hand side: rc(I, J) = sum of r - A z over the aggregate's
// cells, in a fixed order (rows, then columns).
template <bool UNIT>
__global__ void __launch_bounds__(BX *BY) k_restrict(LV L, const float *__restrict__ r, const float *__restrict__ z,
                                                     int cnx, int cny, long long cP, float *__restrict__ rc) {
  auto zf = [&](int xx, int yy) { return z[(long long)yy * L.P + xx]; };
  for (int J = blockIdx.y * BY + threadIdx.y; J < cny; J += gridDim.y * BY)
    for (int I = blockIdx.x * BX + threadIdx.x; I < cnx; I += gridDim.x * BX) {
      float acc = 0.0f;
      for (int dy = 0; dy < 2; dy++) {
        const int y = 2 * J + dy;
        if (y >= L.ny) break;
        for (int dx = 0; dx < 2; dx++) {
          const int x = 2 * I + dx;
          if (x >= L.nx) break;
          float c;
          acc += resid<UNIT>(L, x, y, r[(long long)y * L.P + x], zf, c);
        }
      }
      rc[(long long)J * cP + I] = acc;
    }
}

// The coarsest level (at most kCoarsest x kCoarsest cells, one per thread of
// one CTA): `sweeps` damped-Jacobi sweeps from z = 0 in shared memory. With
// IO64 the level is level 0: r is read from and z written to the FP64 fields.
template <bool UNIT, bool IO64>
__global__ void __launch_bounds__(kCoarseThreads) k_coarsest(LV L, const float *__restrict__ r32,
                                                             const double *__restrict__ r64, long long fp,
                                                             float *__restrict__ zout, double *__restrict__ z64,
                                                             int sweeps, float omega) {
  __shared__ float zs[2][kCoarseThreads];
  const int t = threadIdx.x, n = L.nx * L.ny;
  const bool on = t < n;
  const int x = on ? t % L.nx : 0, y = on ? t / L.nx : 0;
  const long long i = (long long)y * L.P + x;
  float aw = 0.f, ae = 0.f, as = 0.f, an = 0.f, c = 1.f, rv = 0.f;
  if (on) {
    aw = L.ax[i];
    ae = L.ax[i + 1];
    as = L.ay[i];
    an = L.ay[i + L.P];
    c = diag<UNIT>(L, i, aw, ae, as, an);
    rv = IO64 ? (float)r64[(long long)y * fp + x] : r32[i];
  }
  float v = on ? omega * rv / c : 0.f;
  zs[0][t] = v;
  __syncthreads();
  int cur = 0;
  for (int k = 1; k < sweeps; k++) {
    if (on) {
      const float *zc = zs[cur];
      float s = rv - c * zc[t];
      if (x > 0) s += aw * zc[t - 1];
      if (x < L.nx - 1) s += ae * zc[t + 1];
      if (y > 0) s += as * zc[t - L.nx];
      if (y < L.ny - 1) s += an * zc[t + L.nx];
      v = zc[t] + omega * s / c;
    }
    zs[cur ^ 1][t] = v;
    __syncthreads();
    cur ^= 1;
  }
  if (on) {
    if (IO64) z64[(long long)y * fp + x] = (double)v;
    else zout[i] = v;
  }
}

// Level-0 face weights: ax(x, y) = rx Kx[y fp + x] for x in [0, nx],
// ay(x, y) = ry Ky[y fp + x] for y in [0, ny], rounded to FP32.
__global__ void k_fine_faces(int nx, int ny, long long fp, const double *__restrict__ Kx,
                             const double *__restrict__ Ky, double rx, double ry, long long P, float *__restrict__ ax,
                             float *__restrict__ ay) {
  for (int y = blockIdx.y * BY + threadIdx.y; y <= ny; y += gridDim.y * BY)
    for (int x = blockIdx.x * BX + threadIdx.x; x <= nx; x += gridDim.x * BX) {
      const long long s = (long long)y * fp + x, d = (long long)y * P + x;
      if (y < ny) ax[d] = (float)(rx * Kx[s]);
      if (x < nx) ay[d] = (float)(ry * Ky[s]);
    }
}

// Coarse level from fine level F: mass sums, and coarse face I of a row takes
// fine face min(2 I, nx_f) of the aggregate's rows (likewise in y), summed and
// scaled by `fs`.
__global__ void k_coarsen(LV F, int cnx, int cny, long long cP, float *__restrict__ m, float *__restrict__ ax,
                          float *__restrict__ ay, float fs) {
  for (int J = blockIdx.y * BY + threadIdx.y; J <= cny; J += gridDim.y * BY)
    for (int I = blockIdx.x * BX + threadIdx.x; I <= cnx; I += gridDim.x * BX) {
      const long long d = (long long)J * cP + I;
      if (I < cnx && J < cny) {
        float s = 0.f;
        for (int y = 2 * J; y < min(2 * J + 2, F.ny); y++)
          for (int x = 2 * I; x < min(2 * I + 2, F.nx); x++) s += F.m ? F.m[(long long)y * F.P + x] : 1.0f;
        m[d] = s;
      }
      if (J < cny) {
        const int fx = min(2 * I, F.nx);
        float s = 0.f;
        for (int y = 2 * J; y < min(2 * J + 2, F.ny); y++) s += F.ax[(long long)y * F.P + fx];
        ax[d] = fs * s;
      }
      if (I < cnx) {
        const int fy = min(2 * J, F.ny);
        float s = 0.f;
        for (int x = 2 * I; x < min(2 * I + 2, F.nx); x++) s += F.ay[(long long)fy * F.P + x];
        ay[d] = fs * s;
      }
    }
}

}  // namespace

Multigrid::~Multigrid() { release(); }

void Multigrid::drop_graph() {
  if (exec_) cudaGraphExecDestroy(exec_);
  exec_ = nullptr;
  g_r_ = nullptr;
  g_z_ = nullptr;
  g_s_ = nullptr;
}

void Multigrid::release() {
  drop_graph();
  cudaFree(buf_);
  buf_ = nullptr;
  buf_elems_ = 0;
  lv_.clear();
}

void Multigrid::setup(int nx, int ny, long long pitch, const double *Kx, const double *Ky, double rx, double ry,
                      cudaStream_t s) {
  if (nx < 1 || ny < 1 || pitch < nx + 2) throw Error(E_ARG, "multigrid: bad shape");
  // level shapes and storage
  std::vector<Level> lv;
  size_t elems = 0;
  for (int x = nx, y = ny;;) {
    Level L;
    L.nx = x;
    L.ny = y;
    L.pitch = ((long long)x + 1 + 31) / 32 * 32;
    lv.push_back(L);
    const size_t one = (size_t)y * L.pitch;
    elems += 6 * one + L.pitch;  // m (unused on level 0), ax, ay (+1 row), r, z0, z1
    if (x <= kCoarsest && y <= kCoarsest) break;
    x = (x + 1) / 2;
    y = (y + 1) / 2;
  }
  if (lv.size() != lv_.size() || lv[0].nx != (lv_.empty() ? -1 : lv_[0].nx) ||
      lv[0].ny != (lv_.empty() ? -1 : lv_[0].ny) || elems > buf_elems_ || pitch != fpitch_) {
    release();
    OPSB_CUDA(cudaMalloc(&buf_, elems * sizeof(float)));
    buf_elems_ = elems;
    // the cycle never reads the padding columns; they are zeroed once so
    // that every word of the storage is defined
    OPSB_CUDA(cudaMemsetAsync(buf_, 0, elems * sizeof(float), s));
  }
  float *q = buf_;
  for (size_t l = 0; l < lv.size(); l++) {
    Level &L = lv[l];
    const size_t one = (size_t)L.ny * L.pitch;
    L.m = l ? q : nullptr;
    q += one;
    L.ax = q;
    q += one;
    L.ay = q;
    q += one + L.pitch;
    L.r = q;
    q += one;
    L.z0 = q;
    q += one;
    L.z1 = q;
    q += one;
  }
  lv_ = lv;
  fpitch_ = pitch;
  {
    const Level &L = lv_[0];
    k_fine_faces<<<grid_of(nx + 1, ny + 1), dim3(BX, BY), 0, s>>>(nx, ny, pitch, Kx, Ky, rx, ry, L.pitch, L.ax,
                                                                   L.ay);
    check("level-0 faces");
  }
  for (size_t l = 1; l < lv_.size(); l++) {
    const Level &F = lv_[l - 1], &C = lv_[l];
    const LV fv{F.nx, F.ny, F.pitch, F.m, F.ax, F.ay};
    k_coarsen<<<grid_of(C.nx + 1, C.ny + 1), dim3(BX, BY), 0, s>>>(fv, C.nx, C.ny, C.pitch, C.m, C.ax, C.ay,
                                                                    kFaceScale);
    check("coarsening");
  }
}

long long Multigrid::apply(const double *r, double *z, cudaStream_t s) {
  if (lv_.empty()) throw Error(E_STATE, "multigrid: apply before setup");
  if (exec_ && r == g_r_ && z == g_z_ && s == g_s_) {
    OPSB_CUDA(cudaGraphLaunch(exec_, s));
    return g_n_;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  OPSB_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone) return enqueue(r, z, s);  // the caller's capture records the launches
  drop_graph();
  OPSB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  long long n = 0;
  cudaGraph_t g = nullptr;
  try {
    n = enqueue(r, z, s);
  } catch (...) {
    cudaStreamEndCapture(s, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  OPSB_CUDA(cudaStreamEndCapture(s, &g));
  cudaGraphExec_t ex = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  OPSB_CUDA(e);
  exec_ = ex;
  g_r_ = r;
  g_z_ = z;
  g_s_ = s;
  g_n_ = n;
  OPSB_CUDA(cudaGraphLaunch(exec_, s));
  return n;
}

long long Multigrid::enqueue(const double *r, double *z, cudaStream_t s) {
  const int nl = (int)lv_.size();
  const float w = kOmega;
  const dim3 blk(BX, BY);
  auto view = [&](int l) {
    const Level &L = lv_[l];
    return LV{L.nx, L.ny, L.pitch, L.m, L.ax, L.ay};
  };
  long long n = 0;
  if (nl == 1) {
    k_coarsest<true, true><<<1, kCoarseThreads, 0, s>>>(view(0), nullptr, r, fpitch_, nullptr, z, kCoarseSweeps, w);
    check("coarsest level");
    return 1;
  }
  std::vector<float *> zc(nl), out(nl);
  // down: smooth, then hand the residual to the next level
  for (int l = 0; l + 1 < nl; l++) {
    Level &L = lv_[l];
    const LV v = view(l);
    const dim3 g = grid_of(L.nx, L.ny);
    if (l == 0) k_pre_first<true, true><<<g, blk, 0, s>>>(v, r, fpitch_, L.r, L.z0, w);
    else k_pre_first<false, false><<<g, blk, 0, s>>>(v, nullptr, 0, L.r, L.z0, w);
    n++;
    float *cur = L.z0, *oth = L.z1;
    for (int k = 1; k < kSweeps; k++) {
      if (l == 0) k_smooth<true, false><<<g, blk, 0, s>>>(v, L.r, cur, oth, nullptr, 0, w);
      else k_smooth<false, false><<<g, blk, 0, s>>>(v, L.r, cur, oth, nullptr, 0, w);
      n++;
      std::swap(cur, oth);
    }
    zc[l] = cur;
    const Level &C = lv_[l + 1];
    const dim3 gc = grid_of(C.nx, C.ny);
    if (l == 0) k_restrict<true><<<gc, blk, 0, s>>>(v, L.r, cur, C.nx, C.ny, C.pitch, C.r);
    else k_restrict<false><<<gc, blk, 0, s>>>(v, L.r, cur, C.nx, C.ny, C.pitch, C.r);
    n++;
    check("restriction");
  }
  {
    Level &L = lv_[nl - 1];
    k_coarsest<false, false><<<1, kCoarseThreads, 0, s>>>(view(nl - 1), L.r, nullptr, 0, L.z1, nullptr,
                                                          kCoarseSweeps, w);
    n++;
    out[nl - 1] = L.z1;
    check("coarsest level");
  }
  // up: correct with the coarse solution, then post-smooth
  for (int l = nl - 2; l >= 0; l--) {
    Level &L = lv_[l];
    const LV v = view(l);
    const dim3 g = grid_of(L.nx, L.ny);
    const float *e = out[l + 1];
    const long long eP = lv_[l + 1].pitch;
    float *cur = zc[l], *oth = (cur == L.z0) ? L.z1 : L.z0;
    const bool last_first = kSweeps == 1;
    if (l == 0 && last_first) k_post_first<true, true><<<g, blk, 0, s>>>(v, L.r, cur, e, eP, nullptr, z, fpitch_, w);
    else if (l == 0) k_post_first<true, false><<<g, blk, 0, s>>>(v, L.r, cur, e, eP, oth, nullptr, 0, w);
    else k_post_first<false, false><<<g, blk, 0, s>>>(v, L.r, cur, e, eP, oth, nullptr, 0, w);
    n++;
    std::swap(cur, oth);
    for (int k = 1; k < kSweeps; k++) {
      const bool last = k == kSweeps - 1;
      if (l == 0 && last) k_smooth<true, true><<<g, blk, 0, s>>>(v, L.r, cur, nullptr, z, fpitch_, w);
      else if (l == 0) k_smooth<true, false><<<g, blk, 0, s>>>(v, L.r, cur, oth, nullptr, 0, w);
      else k_smooth<false, false><<<g, blk, 0, s>>>(v, L.r, cur, oth, nullptr, 0, w);
      n++;
      std::swap(cur, oth);
    }
    out[l] = cur;
    check("prolongation / post-smoothing");
  }
  return n;
}

}  // namespace heat
}  // namespace opsb
