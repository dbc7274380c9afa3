// extern "C" entry points of include/ops_b200.h over the C++ runtime.
#include <time.h>
#include "../../include/ops_b200.h"

#include <cstddef>
#include <cstring>
#include <string>

#include "runtime.h"

namespace {
thread_local std::string g_last_error = "no error";

template <class F>
int guarded(F &&f) {
  try {
    return f();
  } catch (const opsb::Error &e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return OPS_B200_ERR_STATE;
  } catch (...) {
    g_last_error = "unknown exception";
    return OPS_B200_ERR_STATE;
  }
}

opsb::Runtime &rt() {
  if (!opsb::Runtime::exists()) throw opsb::Error(opsb::E_STATE, "ops_b200_init has not been called");
  return opsb::Runtime::get();
}

std::vector<opsb::Arg> convert_args(int nargs, const ops_b200_arg *args) {
  std::vector<opsb::Arg> out;
  if (nargs < 0 || nargs > OPSB_MAX_ARGS) throw opsb::Error(opsb::E_ARG, "bad argument count");
  for (int i = 0; i < nargs; i++) {
    const ops_b200_arg &a = args[i];
    switch (a.argtype) {
      case OPS_B200_ARG_DAT:
        out.push_back(opsb::arg_dat_opt(a.dat, a.dim, a.stencil, a.acc, a.opt));
        break;
      case OPS_B200_ARG_GBL:
        if (!a.gbl || a.dim <= 0 || a.elem_size <= 0) throw opsb::Error(opsb::E_ARG, "bad global argument");
        out.push_back(opsb::arg_gbl(a.gbl, a.dim, a.elem_size, a.acc));
        break;
      case OPS_B200_ARG_REDUCE:
        out.push_back(opsb::arg_reduce(a.reduction, a.dim, a.acc));
        break;
      case OPS_B200_ARG_IDX:
        out.push_back(opsb::arg_idx());
        break;
      default:
        throw opsb::Error(opsb::E_ARG, "unknown argument type");
    }
  }
  return out;
}
}  // namespace

namespace opsb {
namespace trid {
void set_warp_mode(int m);
}
void set_fcg_chunks(int on);
}  // namespace opsb

extern "C" {

const char *ops_b200_last_error(void) { return g_last_error.c_str(); }

int ops_b200_init(int device, int diags) {
  return guarded([&] {
    opsb::Runtime::get().init(device, diags);
    return 0;
  });
}

int ops_b200_exit(void) {
  return guarded([&] {
    opsb::Runtime::destroy();
    return 0;
  });
}

int ops_b200_decl_block(int dims, const char *name) {
  return guarded([&] { return rt().decl_block(dims, name); });
}

int ops_b200_decl_dat(int block, int dim, const int *size, const int *base, const int *d_m, const int *d_p,
                      const void *data, int type_size, const char *type, const char *name) {
  return guarded([&] {
    if (!size || !d_m || !d_p) throw opsb::Error(opsb::E_ARG, "size, d_m and d_p are required");
    return rt().decl_dat(block, dim, size, base, d_m, d_p, data, type_size, type, name);
  });
}

int ops_b200_decl_stencil(int dims, int points, const int *stencil, const char *name) {
  return guarded([&] {
    if (!stencil) throw opsb::Error(opsb::E_ARG, "stencil offsets required");
    return rt().decl_stencil(dims, points, stencil, nullptr, name);
  });
}

int ops_b200_decl_strided_stencil(int dims, int points, const int *stencil, const int *stride, const char *name) {
  return guarded([&] {
    if (!stencil) throw opsb::Error(opsb::E_ARG, "stencil offsets required");
    return rt().decl_stencil(dims, points, stencil, stride, name);
  });
}

int ops_b200_decl_restrict_stencil(int dims, int points, const int *stencil, const int *stride, const char *name) {
  return guarded([&] {
    if (!stencil) throw opsb::Error(opsb::E_ARG, "stencil offsets required");
    return rt().decl_mgrid_stencil(dims, points, stencil, stride, 2, name);
  });
}

int ops_b200_decl_prolong_stencil(int dims, int points, const int *stencil, const int *stride, const char *name) {
  return guarded([&] {
    if (!stencil) throw opsb::Error(opsb::E_ARG, "stencil offsets required");
    return rt().decl_mgrid_stencil(dims, points, stencil, stride, 1, name);
  });
}

int ops_b200_decl_reduction_handle(int size, const char *type, const char *name) {
  return guarded([&] { return rt().decl_reduction(size, type, name); });
}

int ops_b200_decl_halo(int from, int to, const int *iter_size, const int *from_base, const int *to_base,
                       const int *from_dir, const int *to_dir) {
  return guarded([&] { return rt().decl_halo(from, to, iter_size, from_base, to_base, from_dir, to_dir); });
}

int ops_b200_decl_halo_group(int nhalos, const int *halos) {
  return guarded([&] { return rt().decl_halo_group(nhalos, halos); });
}

int ops_b200_halo_transfer(int group) {
  return guarded([&] {
    rt().halo_transfer(group);
    return 0;
  });
}

int ops_b200_loops_skipped(long long *skipped) {
  return guarded([&] {
    if (skipped) *skipped = rt().loops_skipped();
    return 0;
  });
}

int ops_b200_timers(double *cpu, double *et) {
  return guarded([&] {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    if (et) *et = (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
    clock_gettime(CLOCK_PROCESS_CPUTIME_ID, &ts);
    if (cpu) *cpu = (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
    return 0;
  });
}

int ops_b200_decl_const(const char *name, int dim, const char *type, const void *data) {
  return guarded([&] {
    if (!name || !data) throw opsb::Error(opsb::E_ARG, "constant name and data required");
    rt().decl_const(name, dim, type, data);
    return 0;
  });
}

int ops_b200_update_const(const char *name, int dim, const char *type, const void *data) {
  return ops_b200_decl_const(name, dim, type, data);
}

int ops_b200_par_loop(const char *kernel, const char *name, int block, int dim, const int *range, int nargs,
                      const ops_b200_arg *args) {
  return guarded([&] {
    if (!kernel || !range || (nargs > 0 && !args)) throw opsb::Error(opsb::E_ARG, "kernel, range and args required");
    const opsb::LoopInfo *li = opsb::Runtime::find_loop(kernel);
    if (!li) throw opsb::Error(opsb::E_NOTFOUND, std::string("no registered loop kernel named ") + kernel);
    std::vector<opsb::Arg> a = convert_args(nargs, args);
    rt().par_loop(li, name, block, dim, range, a.data(), (int)a.size());
    return 0;
  });
}

int ops_b200_has_kernel(const char *kernel) { return kernel && opsb::Runtime::find_loop(kernel) ? 1 : 0; }

int ops_b200_execute(void) {
  return guarded([&] {
    rt().execute();
    return 0;
  });
}

int ops_b200_reduction_result(int handle, void *out) {
  return guarded([&] {
    if (!out) throw opsb::Error(opsb::E_ARG, "output pointer required");
    rt().reduction_result(handle, out);
    return 0;
  });
}

int ops_b200_dat_set_data(int dat, const void *data, size_t bytes) {
  return guarded([&] {
    if (!data) throw opsb::Error(opsb::E_ARG, "data pointer required");
    rt().dat_set_data(dat, data, bytes);
    return 0;
  });
}

int ops_b200_dat_fetch_data(int dat, void *data, size_t bytes) {
  return guarded([&] {
    if (!data) throw opsb::Error(opsb::E_ARG, "data pointer required");
    rt().dat_fetch_data(dat, data, bytes);
    return 0;
  });
}

int ops_b200_dat_get_extents(int dat, int *disp, int *size) {
  return guarded([&] {
    rt().dat_get_extents(dat, disp, size);
    return 0;
  });
}

int ops_b200_dat_get_raw_pointer(int dat, int memspace, void **ptr, int *stride) {
  return guarded([&] {
    if (!ptr) throw opsb::Error(opsb::E_ARG, "ptr required");
    if (memspace != OPS_B200_HOST && memspace != OPS_B200_DEVICE) throw opsb::Error(opsb::E_ARG, "bad memspace");
    *ptr = rt().dat_get_raw_pointer(dat, memspace, stride);
    return 0;
  });
}

int ops_b200_dat_release_raw_data(int dat, int acc) {
  return guarded([&] {
    rt().dat_release_raw_data(dat, acc);
    return 0;
  });
}

int ops_b200_set_option(const char *name, int value) {
  return guarded([&] {
    std::string n = name ? name : "";
    if (n == "graphs") rt().set_graphs(value);
    else if (n == "fusion") rt().set_fusion(value);
    else if (n == "tiling") rt().set_tiling(value);
    else if (n == "lists") rt().set_lists(value);
    else if (n == "tile_candidate") rt().set_tile_candidate(value);
    else if (n == "trid_warp") opsb::trid::set_warp_mode(value);
    else if (n == "fcg_chunks") opsb::set_fcg_chunks(value);
    else throw opsb::Error(opsb::E_ARG, "unknown option " + n);
    return 0;
  });
}

int ops_b200_counters(long long *kernels, long long *graphs, long long *loops) {
  return guarded([&] {
    opsb::Runtime &r = rt();
    if (kernels) *kernels = r.kernels_launched();
    if (graphs) *graphs = r.graphs_launched();
    if (loops) *loops = r.loops_enqueued();
    return 0;
  });
}

int ops_b200_fusion_stats(long long *chains, long long *loops, double *fused_bytes, double *loop_bytes) {
  return guarded([&] {
    const opsb::Runtime::FusionStats &s = rt().fusion_stats();
    if (chains) *chains = s.chains;
    if (loops) *loops = s.loops;
    if (fused_bytes) *fused_bytes = s.bytes;
    if (loop_bytes) *loop_bytes = s.loop_bytes;
    return 0;
  });
}

// ---- decomposition across processes ----------------------------------------
namespace {
static_assert(sizeof(ops_b200_msg) == sizeof(opsb::Msg) && offsetof(ops_b200_msg, send) == offsetof(opsb::Msg, send) &&
                  offsetof(ops_b200_msg, recv_bytes) == offsetof(opsb::Msg, recv_bytes),
              "ops_b200_msg and opsb::Msg must share a layout");
struct CCallbacks {
  ops_b200_exchange_fn exchange = nullptr;
  ops_b200_allgather_fn allgather = nullptr;
  void *ctx = nullptr;
};
CCallbacks g_host_cb;  // one transport per process
int host_exchange(void *c, const opsb::Msg *m, int n) {
  const CCallbacks *cb = static_cast<const CCallbacks *>(c);
  return cb->exchange(cb->ctx, reinterpret_cast<const ops_b200_msg *>(m), n);
}
int host_allgather(void *c, const void *send, size_t bytes, void *recv) {
  const CCallbacks *cb = static_cast<const CCallbacks *>(c);
  return cb->allgather(cb->ctx, send, bytes, recv);
}
}  // namespace

int ops_b200_set_transport_host(int nranks, int rank, ops_b200_exchange_fn exchange, ops_b200_allgather_fn allgather,
                                void *ctx) {
  return guarded([&] {
    if (!exchange || !allgather) throw opsb::Error(opsb::E_ARG, "ops_b200_set_transport_host: callbacks required");
    opsb::Runtime &r = opsb::Runtime::get();
    g_host_cb.exchange = exchange;
    g_host_cb.allgather = allgather;
    g_host_cb.ctx = ctx;
    opsb::HostCallbacks hc;
    hc.exchange = host_exchange;
    hc.allgather = host_allgather;
    hc.ctx = &g_host_cb;
    r.set_transport(opsb::make_host_transport(nranks, rank, hc));
    return 0;
  });
}

int ops_b200_nccl_unique_id(void *id128) {
  return guarded([&] {
    if (!id128) throw opsb::Error(opsb::E_ARG, "ops_b200_nccl_unique_id: NULL buffer");
    opsb::nccl_unique_id(id128);
    return 0;
  });
}

int ops_b200_set_transport_nccl(const void *id128, int nranks, int rank) {
  return guarded([&] {
    opsb::Runtime &r = rt();
    OPSB_CUDA(cudaSetDevice(r.device()));
    r.set_transport(opsb::make_nccl_transport(id128, nranks, rank));
    return 0;
  });
}

int ops_b200_partition(const char *routine) {
  return guarded([&] {
    // one process: nothing to split (needs no device, like the reference's
    // single-process ops_partition)
    if (opsb::Runtime::get().nranks() <= 1) return 0;
    rt().partition(routine ? routine : "");
    return 0;
  });
}

int ops_b200_rank_info(int *rank, int *nranks, long long *exchanges) {
  return guarded([&] {
    opsb::Runtime &r = opsb::Runtime::get();
    if (rank) *rank = r.rank();
    if (nranks) *nranks = r.nranks();
    if (exchanges) *exchanges = r.exchanges();
    return 0;
  });
}

int ops_b200_block_slab(int block, int *split_dim, int *extent, int *lo, int *hi, int *halo) {
  return guarded([&] {
    opsb::Runtime &r = rt();
    r.block(block);
    const opsb::Slab &s = r.slab(block);
    if (split_dim) *split_dim = s.dim;
    if (extent) *extent = s.extent;
    if (lo) *lo = s.lo;
    if (hi) *hi = s.hi;
    if (halo) *halo = s.halo;
    return 0;
  });
}

int ops_b200_slab_window(int extent, int nranks, int rank, int halo, int gstart, int gend, int *lo, int *hi,
                         int *own_lo, int *own_hi, int *win_lo, int *win_hi) {
  return guarded([&] {
    if (nranks < 1 || rank < 0 || rank >= nranks || extent < 0 || halo < 0 || gend < gstart)
      throw opsb::Error(opsb::E_ARG, "ops_b200_slab_window: bad arguments");
    opsb::Slab s;
    s.dim = 0;
    s.extent = extent;
    s.halo = halo;
    s.first = rank == 0;
    s.last = rank == nranks - 1;
    opsb::slab_bounds(extent, nranks, rank, &s.lo, &s.hi);
    int a, b, c, d;
    opsb::slab_window(s, gstart, gend, &a, &b, &c, &d);
    if (lo) *lo = s.lo;
    if (hi) *hi = s.hi;
    if (own_lo) *own_lo = a;
    if (own_hi) *own_hi = b;
    if (win_lo) *win_lo = c;
    if (win_hi) *win_hi = d;
    return 0;
  });
}

int ops_b200_transport_selftest(void) {
  return guarded([&] {
    opsb::Transport *t = opsb::Runtime::get().transport();
    if (!t || t->device()) throw opsb::Error(opsb::E_STATE, "transport self-test: no host transport set");
    const int N = t->nranks(), R = t->rank();
    constexpr int kN = 16;
    std::vector<double> out(2 * kN), in(2 * kN, -1.0);
    std::vector<opsb::Msg> msgs;
    for (int side = 0; side < 2; side++) {
      const int peer = side == 0 ? R - 1 : R + 1;
      if (peer < 0 || peer >= N) continue;
      for (int i = 0; i < kN; i++) out[side * kN + i] = R * 1000.0 + peer * 10.0 + i;
      opsb::Msg m;
      m.peer = peer;
      m.send = &out[side * kN];
      m.send_bytes = kN * sizeof(double);
      m.recv = &in[side * kN];
      m.recv_bytes = kN * sizeof(double);
      msgs.push_back(m);
    }
    t->exchange(msgs.data(), (int)msgs.size(), nullptr);
    for (const opsb::Msg &m : msgs) {
      const double *v = static_cast<const double *>(m.recv);
      for (int i = 0; i < kN; i++)
        if (v[i] != m.peer * 1000.0 + R * 10.0 + i)
          throw opsb::Error(opsb::E_STATE, "transport self-test: wrong data from rank " + std::to_string(m.peer));
    }
    std::vector<int> all(N, -1);
    t->allgather(&R, sizeof(int), all.data(), nullptr);
    for (int q = 0; q < N; q++)
      if (all[q] != q) throw opsb::Error(opsb::E_STATE, "transport self-test: allgather out of rank order");
    return 0;
  });
}

int ops_b200_release_spare_storage(long long *freed) {
  return guarded([&] {
    long long n = (long long)rt().release_spare_storage();
    if (freed) *freed = n;
    return 0;
  });
}

int ops_b200_tridsolver_params_init(ops_b200_tridsolver_params *p, int block, int strategy) {
  return guarded([&] {
    if (!p) throw opsb::Error(opsb::E_ARG, "ops_tridsolver_params: NULL params");
    if (strategy < -1 || strategy > 5) throw opsb::Error(opsb::E_ARG, "ops_tridsolver_params: unknown strategy");
    std::memset(p, 0, sizeof(*p));
    p->block = block;
    p->strategy = strategy < 0 ? 0 : strategy;
    return 0;
  });
}

int ops_b200_tridsolver_params_set_jacobi_params(ops_b200_tridsolver_params *p, double rtol, double atol,
                                                 int maxiter) {
  return guarded([&] {
    if (!p || !(rtol >= 0.0) || !(atol >= 0.0) || maxiter < 0)
      throw opsb::Error(opsb::E_ARG, "set_jacobi_params: tolerances and maxiter must be non-negative");
    p->jacobi_rtol = rtol;
    p->jacobi_atol = atol;
    p->jacobi_maxiter = maxiter;
    return 0;
  });
}

int ops_b200_tridsolver_params_set_batch_size(ops_b200_tridsolver_params *p, int batch_size) {
  return guarded([&] {
    if (!p || batch_size < 0) throw opsb::Error(opsb::E_ARG, "set_batch_size: batch size must be non-negative");
    p->batch_size = batch_size;
    return 0;
  });
}

int ops_b200_tridsolver_params_set_cuda_opts(ops_b200_tridsolver_params *p, int opt_x, int opt_y, int opt_z) {
  return guarded([&] {
    if (!p) throw opsb::Error(opsb::E_ARG, "set_cuda_opts: NULL params");
    p->cuda_opts[0] = opt_x;
    p->cuda_opts[1] = opt_y;
    p->cuda_opts[2] = opt_z;
    return 0;
  });
}

int ops_b200_tridsolver_params_set_cuda_sync(ops_b200_tridsolver_params *p, int sync) {
  return guarded([&] {
    if (!p) throw opsb::Error(opsb::E_ARG, "set_cuda_sync: NULL params");
    p->cuda_sync = sync;
    return 0;
  });
}

int ops_b200_reset_counters(void) {
  return guarded([&] {
    rt().reset_counters();
    rt().reset_fusion_stats();
    return 0;
  });
}

int ops_b200_set_kernel_timing(int on) {
  return guarded([&] {
    rt().set_timing(on);
    return 0;
  });
}

int ops_b200_kernel_time(const char *kernel, long long *launches, double *total_ms) {
  return guarded([&] {
    const auto &m = rt().kernel_times();
    auto it = m.find(kernel ? kernel : "");
    if (launches) *launches = it == m.end() ? 0 : it->second.launches;
    if (total_ms) *total_ms = it == m.end() ? 0.0 : it->second.ms;
    return 0;
  });
}

int ops_b200_kernel_stats(ops_b200_kernel_stat *out, int max) {
  return guarded([&] {
    const auto &m = rt().kernel_times();
    int n = 0;
    for (const auto &kv : m) {
      if (out && n < max) {
        strncpy(out[n].name, kv.first.c_str(), sizeof(out[n].name) - 1);
        out[n].name[sizeof(out[n].name) - 1] = 0;
        out[n].launches = kv.second.launches;
        out[n].total_ms = kv.second.ms;
        out[n].alg_bytes = kv.second.bytes;
      }
      n++;
    }
    return n;
  });
}

int ops_b200_clear_kernel_timing(void) {
  return guarded([&] {
    rt().clear_timing();
    return 0;
  });
}

}  // extern "C"

// App entry points are defined next to their drivers (apps_*.cpp) and use
// this helper to share the error path.
namespace opsb {
int capi_guard(const std::function<int()> &f) { return guarded(f); }
}  // namespace opsb
