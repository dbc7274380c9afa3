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

// ---------------------------------------------------------------------------
// raw heat solves and the learned preconditioner's network handles
// ---------------------------------------------------------------------------
#include <memory>
#include <vector>

#include "heat_pcg.h"
#include "heat_mg.h"
#include "lmg.h"

namespace opsb {
namespace {

struct HeatWorkspace {
  int nx = 0, ny = 0;
  long long pitch = 0;
  double *buf = nullptr;
  double *r = nullptr, *w = nullptr, *p = nullptr, *z = nullptr, *Mi = nullptr;
  double *t = nullptr;  // the multigrid part of the learned-multigrid preconditioner
  heat::Solver solver;
  heat::Multigrid mg;
  ~HeatWorkspace() { cudaFree(buf); }
  void ensure(int x, int y, long long pt, cudaStream_t s) {
    if (x == nx && y == ny && pt == pitch && buf) return;
    cudaFree(buf);
    buf = nullptr;
    const size_t one = (size_t)pt * (y + 2);
    OPSB_CUDA(cudaMalloc(&buf, 6 * one * sizeof(double)));
    OPSB_CUDA(cudaMemsetAsync(buf, 0, 6 * one * sizeof(double), s));
    double **f[6] = {&r, &w, &p, &z, &Mi, &t};
    for (int k = 0; k < 6; k++) *f[k] = buf + k * one + pt + 1;
    nx = x;
    ny = y;
    pitch = pt;
  }
};

// z = z - r / D + t on the interior, D = diag(A) computed as the network
// computes it (lmg.cu `coef`): the network's output r / D + s y becomes the
// correction s y added to the multigrid cycle's t. With an untrained network
// (y = 0) the result is t exactly.
__global__ void k_learned_mg_combine(int nx, int ny, long long pitch, const double *__restrict__ Kx,
                                     const double *__restrict__ Ky, double rx, double ry,
                                     const double *__restrict__ r, const double *__restrict__ t,
                                     double *__restrict__ z) {
  for (int y = blockIdx.y * blockDim.y + threadIdx.y; y < ny; y += gridDim.y * blockDim.y)
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < nx; x += gridDim.x * blockDim.x) {
      const long long i = (long long)y * pitch + x;
      const double a = rx * Kx[i], b = rx * Kx[i + 1], c = ry * Ky[i], d = ry * Ky[i + pitch];
      const double D = 1.0 + a + b + c + d;
      z[i] = (z[i] - r[i] / D) + t[i];
    }
}

std::mutex g_mu;
cudaStream_t own_stream() {
  static cudaStream_t st[64] = {nullptr};
  int dev = 0;
  OPSB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw Error(E_CUDA, "device index out of range");
  if (!st[dev]) OPSB_CUDA(cudaStreamCreate(&st[dev]));
  return st[dev];
}
HeatWorkspace &workspace() {
  static HeatWorkspace ws;
  return ws;
}
std::vector<std::unique_ptr<lmg::Net>> &nets() {
  static std::vector<std::unique_ptr<lmg::Net>> v;
  return v;
}
lmg::Net &net_of(int h) {
  if (h < 0 || h >= (int)nets().size() || !nets()[h]) throw Error(E_ARG, "unknown learned-preconditioner handle");
  return *nets()[h];
}
lmg::Fields fields_of(const ops_b200_heat_batch *b) {
  if (!b || !b->r || !b->Kx || !b->Ky) throw Error(E_ARG, "heat batch: null field");
  if (b->n < 1 || b->h < 8 || b->w < 8 || b->h % 8 || b->w % 8)
    throw Error(E_ARG, "heat batch: h and w must be positive multiples of 8");
  if (b->pitch < b->w + 2 || (b->n > 1 && b->image < b->pitch * (b->h + 2)))
    throw Error(E_ARG, "heat batch: pitch or image stride too small for a one-cell ring");
  lmg::Fields f;
  f.n = b->n;
  f.h = b->h;
  f.w = b->w;
  f.pitch = b->pitch;
  f.image = b->image;
  f.r = b->r;
  f.Kx = b->Kx;
  f.Ky = b->Ky;
  f.rx = b->rx;
  f.ry = b->ry;
  return f;
}

}  // namespace
}  // namespace opsb

namespace opsb {
namespace {
// The 3D solver's own fields (zero on every halo cell), kept per size.
struct Heat3DWorkspace {
  int nx = 0, ny = 0, nz = 0;
  long long pitch = 0;
  double *buf = nullptr;
  double *r = nullptr, *w = nullptr, *p = nullptr, *z = nullptr, *Mi = nullptr;
  heat::Solver solver;
  ~Heat3DWorkspace() { cudaFree(buf); }
  void ensure(int x, int y, int zz, long long pt, cudaStream_t s) {
    if (x == nx && y == ny && zz == nz && pt == pitch && buf) return;
    cudaFree(buf);
    buf = nullptr;
    nx = ny = nz = 0;
    const size_t one = (size_t)pt * (y + 2) * (zz + 2);
    OPSB_CUDA(cudaMalloc(&buf, 5 * one * sizeof(double)));
    OPSB_CUDA(cudaMemsetAsync(buf, 0, 5 * one * sizeof(double), s));
    const size_t first = (size_t)pt * (y + 2) + pt + 1;
    double **f[5] = {&r, &w, &p, &z, &Mi};
    for (int k = 0; k < 5; k++) *f[k] = buf + k * one + first;
    nx = x;
    ny = y;
    nz = zz;
    pitch = pt;
  }
};
Heat3DWorkspace &workspace3d() {
  static Heat3DWorkspace w;
  return w;
}
}  // namespace

// "fcg_chunks" option: replayed FCG chunks on (default) or the host loop.
bool &fcg_chunks_flag() {
  static bool on = true;
  return on;
}
bool fcg_chunks_on() { return fcg_chunks_flag(); }
void set_fcg_chunks(int on) { fcg_chunks_flag() = on != 0; }
}  // namespace opsb

extern "C" int ops_b200_heat_solve(const ops_b200_heat_system *sys, int method, int net, double eps, int max_iters,
                                   int window, double *r_out, ops_b200_heat_stats *stats, void *stream) {
  using namespace opsb;
  return capi_guard([&] {
    if (!sys || !sys->Kx || !sys->Ky || !sys->u0 || !sys->u) throw Error(E_ARG, "heat system: null field");
    if (sys->nx < 1 || sys->ny < 1 || sys->pitch < sys->nx + 2) throw Error(E_ARG, "heat system: bad shape");
    if (method < OPS_B200_HEAT_PCG || method > OPS_B200_HEAT_FCG_LEARNED_MG) throw Error(E_ARG, "heat system: method");
    if (!(eps > 0.0) || max_iters < 0) throw Error(E_ARG, "heat system: eps > 0 and max_iters >= 0 required");
    std::lock_guard<std::mutex> lk(g_mu);
    // the iteration chunks are replayed from CUDA graphs, which cannot be
    // captured on the legacy NULL stream: a NULL stream means the library's own
    // blocking stream (ordered with the NULL stream both ways)
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!s) s = own_stream();
    HeatWorkspace &ws = workspace();
    ws.ensure(sys->nx, sys->ny, sys->pitch, s);
    heat::Field2D f;
    f.nx = sys->nx;
    f.ny = sys->ny;
    f.pitch = sys->pitch;
    f.Kx = sys->Kx;
    f.Ky = sys->Ky;
    f.u0 = sys->u0;
    f.u = sys->u;
    f.r = ws.r;
    f.w = ws.w;
    f.p = ws.p;
    f.z = ws.z;
    f.Mi = ws.Mi;
    ws.solver.diag(f, sys->rx, sys->ry, s);
    heat::SolveStats st;
    cudaEvent_t e0, e1;
    OPSB_CUDA(cudaEventCreate(&e0));
    OPSB_CUDA(cudaEventCreate(&e1));
    OPSB_CUDA(cudaEventRecord(e0, s));
    if (method == OPS_B200_HEAT_PCG || method == OPS_B200_HEAT_PCG_TRUE) {
      ws.solver.pcg_fp64(f, sys->rx, sys->ry, true, method == OPS_B200_HEAT_PCG_TRUE, eps, max_iters, s, &st);
    } else if (method == OPS_B200_HEAT_MIXED) {
      if (sys->nx < 1) throw Error(E_ARG, "heat system: bad shape");
      ws.solver.pcg_mixed(f, sys->rx, sys->ry, true, eps, 0.1, max_iters, s, &st);
    } else {
      heat::Solver::Precond M, fallback;
      if (method == OPS_B200_HEAT_FCG_LEARNED || method == OPS_B200_HEAT_FCG_LEARNED_MG) {
        lmg::Net *np = &net_of(net);
        if (sys->nx % 8 || sys->ny % 8) throw Error(E_ARG, "learned preconditioner: nx and ny must be multiples of 8");
        lmg::Fields lf;
        lf.n = 1;
        lf.h = sys->ny;
        lf.w = sys->nx;
        lf.pitch = sys->pitch;
        lf.image = 0;
        lf.r = ws.r;
        lf.Kx = sys->Kx;
        lf.Ky = sys->Ky;
        lf.rx = sys->rx;
        lf.ry = sys->ry;
        M = [np, lf](const double *, double *z, cudaStream_t ss) -> long long {
          const long long before = np->launches();
          np->apply(lf, z, ss);
          return np->launches() - before;
        };
        if (method == OPS_B200_HEAT_FCG_LEARNED_MG) {
          heat::Multigrid *mg = &ws.mg;
          mg->setup(sys->nx, sys->ny, sys->pitch, sys->Kx, sys->Ky, sys->rx, sys->ry, s);
          fallback = [mg](const double *r, double *z, cudaStream_t ss) -> long long { return mg->apply(r, z, ss); };
          const heat::Solver::Precond net_part = M;
          const int nx = sys->nx, ny = sys->ny;
          const long long pitch = sys->pitch;
          const double *Kx = sys->Kx, *Ky = sys->Ky, rx = sys->rx, ry = sys->ry;
          double *t = ws.t;
          M = [=](const double *r, double *z, cudaStream_t ss) -> long long {
            long long n = net_part(r, z, ss) + mg->apply(r, t, ss);
            const dim3 blk(128, 2), grd((nx + 127) / 128, std::min((ny + 1) / 2, 4096));
            k_learned_mg_combine<<<grd, blk, 0, ss>>>(nx, ny, pitch, Kx, Ky, rx, ry, r, t, z);
            OPSB_CUDA(cudaGetLastError());
            return n + 1;
          };
        }
      } else if (method == OPS_B200_HEAT_FCG_MG) {
        heat::Multigrid *mg = &ws.mg;
        mg->setup(sys->nx, sys->ny, sys->pitch, sys->Kx, sys->Ky, sys->rx, sys->ry, s);
        M = [mg](const double *r, double *z, cudaStream_t ss) -> long long { return mg->apply(r, z, ss); };
      }
      // the network's application and Jacobi are plain kernel launches, so
      // those solves replay their iterations from graphs; the multigrid
      // variants launch the V-cycle's own graph and keep the host loop
      const bool chunked =
          fcg_chunks_on() && (method == OPS_B200_HEAT_FCG_LEARNED || method == OPS_B200_HEAT_FCG_JACOBI);
      ws.solver.fcg(f, sys->rx, sys->ry, eps, max_iters, M, window, s, &st, fallback ? &fallback : nullptr,
                    chunked);
    }
    OPSB_CUDA(cudaEventRecord(e1, s));
    OPSB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    OPSB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    double fin = st.true_residual;
    if (r_out) fin = ws.solver.residual(f, sys->rx, sys->ry, r_out, s);
    if (method == OPS_B200_HEAT_FCG_LEARNED || method == OPS_B200_HEAT_FCG_LEARNED_MG) {
      int err = 0;
      OPSB_CUDA(cudaMemcpy(&err, cnn::error_word(), sizeof(int), cudaMemcpyDeviceToHost));
      if (err) throw Error(E_TIMEOUT, "learned preconditioner: a convolution pipeline wait expired");
    }
    if (stats) {
      stats->iterations = st.iterations;
      stats->updates = st.outer;
      stats->converged = st.converged;
      stats->fallbacks = st.fallbacks;
      stats->initial_residual = st.initial_residual;
      stats->final_residual = fin;
      stats->seconds = ms * 1e-3;
      stats->launches = ws.solver.launches();
    }
    return 0;
  });
}

extern "C" int ops_b200_heat_mg_apply(const ops_b200_heat_system *sys, const double *r, double *z, int *levels,
                                      void *stream) {
  using namespace opsb;
  return capi_guard([&] {
    if (!sys || !sys->Kx || !sys->Ky || !r || !z) throw Error(E_ARG, "heat multigrid: null field");
    if (sys->nx < 1 || sys->ny < 1 || sys->pitch < sys->nx + 2) throw Error(E_ARG, "heat multigrid: bad shape");
    std::lock_guard<std::mutex> lk(g_mu);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!s) s = own_stream();
    HeatWorkspace &ws = workspace();
    ws.mg.setup(sys->nx, sys->ny, sys->pitch, sys->Kx, sys->Ky, sys->rx, sys->ry, s);
    ws.mg.apply(r, z, s);
    OPSB_CUDA(cudaStreamSynchronize(s));
    if (levels) *levels = ws.mg.levels();
    return 0;
  });
}

extern "C" int ops_b200_lmg_create(unsigned long long seed) {
  using namespace opsb;
  return capi_guard([&] {
    std::lock_guard<std::mutex> lk(g_mu);
    nets().emplace_back(new lmg::Net(seed));
    return (int)nets().size() - 1;
  });
}

extern "C" int ops_b200_lmg_destroy(int net) {
  using namespace opsb;
  return capi_guard([&] {
    std::lock_guard<std::mutex> lk(g_mu);
    net_of(net);
    nets()[net].reset();
    return 0;
  });
}

extern "C" int ops_b200_lmg_num_params(void) { return opsb::lmg::Net::num_params(); }

extern "C" int ops_b200_lmg_get_params(int net, float *host) {
  using namespace opsb;
  return capi_guard([&] {
    if (!host) throw Error(E_ARG, "null buffer");
    net_of(net).get_params(host);
    return 0;
  });
}

extern "C" int ops_b200_lmg_set_params(int net, const float *host) {
  using namespace opsb;
  return capi_guard([&] {
    if (!host) throw Error(E_ARG, "null buffer");
    net_of(net).set_params(host);
    return 0;
  });
}

extern "C" int ops_b200_lmg_get_grads(int net, float *host) {
  using namespace opsb;
  return capi_guard([&] {
    if (!host) throw Error(E_ARG, "null buffer");
    net_of(net).get_grads(host);
    return 0;
  });
}

extern "C" int ops_b200_lmg_apply(int net, const ops_b200_heat_batch *b, double *out, void *stream) {
  using namespace opsb;
  return capi_guard([&] {
    if (!out) throw Error(E_ARG, "null output");
    lmg::Fields f = fields_of(b);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    net_of(net).apply(f, out, s);
    OPSB_CUDA(cudaStreamSynchronize(s));
    int err = 0;
    OPSB_CUDA(cudaMemcpy(&err, cnn::error_word(), sizeof(int), cudaMemcpyDeviceToHost));
    if (err) throw Error(E_TIMEOUT, "learned preconditioner: a convolution pipeline wait expired");
    return 0;
  });
}

extern "C" int ops_b200_lmg_train_step(int net, const ops_b200_heat_batch *b, const double *e, int loss_kind,
                                       double lr, double *loss, void *stream) {
  using namespace opsb;
  return capi_guard([&] {
    if (!e) throw Error(E_ARG, "null target");
    lmg::Fields f = fields_of(b);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    lmg::Net &nt = net_of(net);
    if (loss_kind != lmg::LOSS_L2 && loss_kind != lmg::LOSS_ANORM) throw Error(E_ARG, "loss_kind must be 0 or 1");
    const double L = nt.loss_and_grad(f, e, loss_kind, s);
    if (lr > 0.0) nt.adam(lr, s);
    OPSB_CUDA(cudaStreamSynchronize(s));
    if (loss) *loss = L;
    return 0;
  });
}

extern "C" int ops_b200_heat_solve3d(const ops_b200_heat_system3d *sys, int method, double eps, int max_iters,
                                     ops_b200_heat_stats *stats, void *stream) {
  using namespace opsb;
  return capi_guard([&] {
    if (!sys || !sys->Kx || !sys->Ky || !sys->Kz || !sys->u0 || !sys->u) throw Error(E_ARG, "heat system 3D: null field");
    if (sys->nx < 1 || sys->ny < 1 || sys->nz < 1 || sys->pitch < sys->nx + 2 || sys->plane != sys->pitch * (sys->ny + 2))
      throw Error(E_ARG, "heat system 3D: bad shape (pitch >= nx + 2, plane == pitch * (ny + 2))");
    if (method != OPS_B200_HEAT_PCG && method != OPS_B200_HEAT_PCG_TRUE && method != OPS_B200_HEAT_MIXED)
      throw Error(E_ARG, "heat system 3D: methods OPS_B200_HEAT_PCG, OPS_B200_HEAT_PCG_TRUE and OPS_B200_HEAT_MIXED");
    if (!(eps > 0.0) || max_iters < 0) throw Error(E_ARG, "heat system 3D: eps > 0 and max_iters >= 0 required");
    std::lock_guard<std::mutex> lk(g_mu);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!s) s = own_stream();
    Heat3DWorkspace &ws = workspace3d();
    ws.ensure(sys->nx, sys->ny, sys->nz, sys->pitch, s);
    heat::Field3D f;
    f.nx = sys->nx;
    f.ny = sys->ny;
    f.nz = sys->nz;
    f.pitch = sys->pitch;
    f.plane = sys->plane;
    f.Kx = sys->Kx;
    f.Ky = sys->Ky;
    f.Kz = sys->Kz;
    f.u0 = sys->u0;
    f.u = sys->u;
    f.r = ws.r;
    f.w = ws.w;
    f.p = ws.p;
    f.z = ws.z;
    f.Mi = ws.Mi;
    ws.solver.diag3(f, sys->rx, sys->ry, sys->rz, s);
    heat::SolveStats st;
    cudaEvent_t e0, e1;
    OPSB_CUDA(cudaEventCreate(&e0));
    OPSB_CUDA(cudaEventCreate(&e1));
    OPSB_CUDA(cudaEventRecord(e0, s));
    try {
      if (method == OPS_B200_HEAT_MIXED)
        ws.solver.pcg3d_mixed(f, sys->rx, sys->ry, sys->rz, eps, 0.1, max_iters, s, &st);
      else
        ws.solver.pcg3d(f, sys->rx, sys->ry, sys->rz, method == OPS_B200_HEAT_PCG_TRUE, eps, max_iters, s, &st);
      OPSB_CUDA(cudaEventRecord(e1, s));
      OPSB_CUDA(cudaEventSynchronize(e1));
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
      memset(stats, 0, sizeof(*stats));
      stats->iterations = st.iterations;
      stats->updates = st.outer;
      stats->converged = st.converged;
      stats->initial_residual = st.initial_residual;
      stats->final_residual = st.true_residual;
      stats->seconds = ms * 1e-3;
      stats->launches = ws.solver.launches();
    }
    return 0;
  });
}
