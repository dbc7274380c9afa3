// OPS-B200 host runtime (see runtime.h for the reference mapping).
#include "runtime.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <sstream>

namespace opsb {

void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    std::ostringstream os;
    os << "CUDA error " << cudaGetErrorName(e) << " (" << cudaGetErrorString(e) << ") in " << what;
    throw Error(E_CUDA, os.str());
  }
}

// ---------------------------------------------------------------------------
// Registries (populated at static-initialisation time by the kernel modules).
// ---------------------------------------------------------------------------
namespace {
struct Registry {
  std::map<std::string, std::unique_ptr<LoopInfo>> loops;
  struct ConstSlot { std::string scope; const void *symbol; size_t offset, bytes; };
  std::multimap<std::string, ConstSlot> consts;
  std::vector<ChainRule> chains;
};
Registry &registry() {
  static Registry r;
  return r;
}
Runtime *g_runtime = nullptr;

inline uint64_t mix64(uint64_t h, uint64_t v) {
  // FNV-1a style fold of 64-bit words.
  h ^= v + 0x9E3779B97F4A7C15ULL + (h << 6) + (h >> 2);
  return h * 0x100000001B3ULL;
}

constexpr size_t kGblCap = 1 << 20;
}  // namespace

void Runtime::register_loop(const LoopInfo &info) {
  registry().loops[info.kernel] = std::make_unique<LoopInfo>(info);
}
const LoopInfo *Runtime::find_loop(const std::string &kernel) {
  auto &m = registry().loops;
  auto it = m.find(kernel);
  return it == m.end() ? nullptr : it->second.get();
}
// Constant slots are registered as "<app>/<name>" (the app prefix of the
// kernels that read them) and looked up by <name>.
static void split_const_name(const std::string &q, std::string &scope, std::string &name) {
  size_t k = q.find('/');
  scope = k == std::string::npos ? std::string() : q.substr(0, k);
  name = k == std::string::npos ? q : q.substr(k + 1);
}
void Runtime::register_const(const std::string &qualified, const void *symbol, size_t offset, size_t bytes) {
  std::string scope, name;
  split_const_name(qualified, scope, name);
  registry().consts.insert({name, {scope, symbol, offset, bytes}});
}
void Runtime::register_chain(const ChainRule &rule) { registry().chains.push_back(rule); }

Runtime &Runtime::get() {
  if (!g_runtime) g_runtime = new Runtime();
  return *g_runtime;
}
bool Runtime::exists() { return g_runtime != nullptr && g_runtime->inited_; }
void Runtime::destroy() {
  delete g_runtime;
  g_runtime = nullptr;
}

Runtime::~Runtime() {
  if (!inited_) return;
  cudaStreamSynchronize(stream_);
  for (auto &p : pending_) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  for (auto e : event_pool_) cudaEventDestroy(e);
  for (auto &kv : graphs_)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  release_fusion_state();
  for (auto &kv : shadow_)
    if (kv.second) cudaFree(kv.second);
  for (auto &d : dats_)
    if (d && d->data_d) cudaFree(d->data_d);
  for (auto &kv : spare_) cudaFree(kv.second);
  if (red_arena_) cudaFree(red_arena_);
  if (gbl_dev_) cudaFree(gbl_dev_);
  if (red_scratch_) cudaFree(red_scratch_);
  if (red_counters_) cudaFree(red_counters_);
  if (red_host_) cudaFreeHost(red_host_);
  if (stage_h_) cudaFreeHost(stage_h_);
  for (auto &kv : list_cache_) cudaFree(kv.second);
  transport_.reset();
  if (stream_) cudaStreamDestroy(stream_);
}

void Runtime::init(int device, int diags) {
  if (inited_) return;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    throw Error(E_CUDA, "ops_b200: no CUDA device available (the B200 backend has no CPU path)");
  if (device < 0 || device >= n) throw Error(E_ARG, "ops_b200: device index out of range");
  device_ = device;
  diags_ = diags;
  OPSB_CUDA(cudaSetDevice(device_));
  OPSB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  OPSB_CUDA(cudaMalloc(&gbl_dev_, kGblCap));
  gbl_host_.resize(kGblCap);
  gbl_cap_ = kGblCap;
  size_t scratch = (size_t)OPSB_MAX_REDUCE_ARGS * kMaxRedBlocks * OPSB_MAX_RED_DIM * sizeof(double);
  OPSB_CUDA(cudaMalloc(&red_scratch_, scratch));
  OPSB_CUDA(cudaMalloc(&red_counters_, kNumCounters * sizeof(unsigned int)));
  OPSB_CUDA(cudaMemset(red_counters_, 0, kNumCounters * sizeof(unsigned int)));
  OPSB_CUDA(cudaMalloc(&red_arena_, kRedArenaBytes));
  OPSB_CUDA(cudaMemset(red_arena_, 0, kRedArenaBytes));
  OPSB_CUDA(cudaMallocHost(&red_host_, kRedArenaBytes));
  const char *g = getenv("OPS_B200_GRAPHS");
  if (g) graphs_on_ = atoi(g);
  const char *f = getenv("OPS_B200_FUSION");
  if (f) fusion_on_ = atoi(f);
  const char *t = getenv("OPS_B200_TILING");
  if (t) tiling_on_ = atoi(t);
  const char *l = getenv("OPS_B200_LISTS");
  if (l) lists_on_ = atoi(l);
  const char *tc = getenv("OPS_B200_TILE_CANDIDATE");
  if (tc) set_tile_candidate(atoi(tc));
  inited_ = true;
}

// A checked condition; the message (often built from strings) is evaluated
// only when the check fails, so the checks cost nothing on the loop path.
#define OPSB_REQUIRE(cond, code, msg)              \
  do {                                             \
    if (!(cond)) throw Error((code), (msg));       \
  } while (0)

Dat &Runtime::dat(int i) {
  OPSB_REQUIRE(i >= 0 && i < (int)dats_.size() && dats_[i], E_ARG, "invalid dat handle " + std::to_string(i));
  return *dats_[i];
}
Stencil &Runtime::stencil(int i) {
  OPSB_REQUIRE(i >= 0 && i < (int)stencils_.size(), E_ARG, "invalid stencil handle " + std::to_string(i));
  return stencils_[i];
}
Reduction &Runtime::reduction(int i) {
  OPSB_REQUIRE(i >= 0 && i < (int)reductions_.size(), E_ARG, "invalid reduction handle " + std::to_string(i));
  return reductions_[i];
}
Block &Runtime::block(int i) {
  OPSB_REQUIRE(i >= 0 && i < (int)blocks_.size(), E_ARG, "invalid block handle " + std::to_string(i));
  return blocks_[i];
}

int Runtime::decl_block(int dims, const char *name) {
  OPSB_REQUIRE(inited_, E_STATE, "ops_decl_block before ops_init");
  OPSB_REQUIRE(dims >= 1 && dims <= 3, E_UNSUPPORTED, "blocks of 1 to 3 dimensions are supported");
  Block b;
  b.index = (int)blocks_.size();
  b.dims = dims;
  b.name = name ? name : "";
  blocks_.push_back(b);
  return b.index;
}

static int type_size_of(const char *type) {
  std::string t = type ? type : "";
  if (t == "double" || t == "long" || t == "long long" || t == "ll") return 8;
  if (t == "float" || t == "int" || t == "unsigned int") return 4;
  if (t == "short" || t == "half") return 2;
  if (t == "char") return 1;
  return 0;
}

int Runtime::decl_dat(int blk, int dim, const int *size, const int *base, const int *d_m, const int *d_p,
                      const void *data, int type_size, const char *type, const char *name) {
  OPSB_REQUIRE(inited_, E_STATE, "ops_decl_dat before ops_init");
  Block &b = block(blk);
  OPSB_REQUIRE(dim >= 1, E_ARG, "dat dim must be >= 1");
  int ts = type_size > 0 ? type_size : type_size_of(type);
  OPSB_REQUIRE(ts > 0, E_ARG, std::string("unknown dat type ") + (type ? type : "(null)"));
  auto d = std::make_unique<Dat>();
  d->index = (int)dats_.size();
  d->block = blk;
  d->dim = dim;
  d->type_size = ts;
  d->elem_size = ts * dim;
  d->type = type ? type : "";
  d->name = name ? name : "";
  for (int i = 0; i < 3; i++) {
    if (i < b.dims) {
      OPSB_REQUIRE(d_m[i] <= 0 && d_p[i] >= 0, E_ARG, "halo depths must satisfy d_m <= 0 <= d_p");
      OPSB_REQUIRE(size[i] >= 0, E_ARG, "negative dat size");
      d->base[i] = base ? base[i] : 0;
      d->d_m[i] = d_m[i];
      d->d_p[i] = d_p[i];
      // ops_dat_init_metadata_core (ops/c/src/core/ops_lib_core.cpp:469-474)
      d->size[i] = size[i] - d_m[i] + d_p[i];
    } else {
      d->size[i] = 1;
    }
  }
  // Logical index 0 of x starts on a 64-byte boundary; rows are 128-byte pitched.
  const int e = d->elem_size;
  int lead = -d->d_m[0] + d->base[0] * 0;  // columns before logical x = 0
  int align_elems = (e <= 64 && 64 % e == 0) ? 64 / e : 1;
  d->pad_front = (align_elems - (lead % align_elems)) % align_elems;
  int row_align = (e <= 128 && 128 % e == 0) ? 128 / e : 1;
  d->pitch = ((long long)(d->pad_front + d->size[0]) + row_align - 1) / row_align * row_align;
  d->plane = d->pitch * d->size[1];
  d->origin = d->pad_front + (long long)(-d->base[0] - d->d_m[0]) + (long long)(-d->base[1] - d->d_m[1]) * d->pitch +
              (long long)(-d->base[2] - d->d_m[2]) * d->plane;
  d->bytes = (size_t)d->plane * d->size[2] * e;
  for (int i = 0; i < 3; i++) {
    d->lo[i] = d->own_lo[i] = d->base[i] + d->d_m[i];
    d->hi[i] = d->own_hi[i] = d->lo[i] + d->size[i];
  }
  d->data_d = alloc_dat_storage(d->bytes);
  OPSB_CUDA(cudaMemsetAsync(d->data_d, 0, d->bytes, stream_));
  int idx = d->index;
  dats_.push_back(std::move(d));
  if (data) {
    const Dat &dd = *dats_[idx];
    dat_set_data(idx, data, (size_t)dd.size[0] * dd.size[1] * dd.size[2] * dd.elem_size);
  }
  OPSB_CUDA(cudaStreamSynchronize(stream_));
  // a dat declared on a block already partitioned gets its slab at once
  if (blk < (int)slabs_.size()) window_dat(*dats_[idx]);
  return idx;
}

int Runtime::decl_stencil(int dims, int points, const int *offs, const int *stride, const char *name) {
  OPSB_REQUIRE(inited_, E_STATE, "ops_decl_stencil before ops_init");
  OPSB_REQUIRE(dims >= 1 && dims <= 3 && points >= 1, E_ARG, "bad stencil shape");
  Stencil s;
  s.index = (int)stencils_.size();
  s.dims = dims;
  s.points = points;
  s.offs.assign(offs, offs + (size_t)dims * points);
  for (int i = 0; i < 3; i++) s.stride[i] = (stride && i < dims) ? stride[i] : 1;
  s.name = name ? name : "";
  stencils_.push_back(s);
  return s.index;
}

int Runtime::decl_mgrid_stencil(int dims, int points, const int *offs, const int *mgrid_stride, int type,
                                const char *name) {
  OPSB_REQUIRE(type == 1 || type == 2, E_ARG, "multigrid stencil type must be 1 (prolong) or 2 (restrict)");
  OPSB_REQUIRE(mgrid_stride != nullptr, E_ARG, "multigrid stencils need a stride");
  for (int i = 0; i < dims && i < 3; i++) OPSB_REQUIRE(mgrid_stride[i] >= 1, E_ARG, "multigrid stride must be >= 1");
  int h = decl_stencil(dims, points, offs, nullptr, name);
  Stencil &st = stencils_[h];
  st.type = type;
  for (int i = 0; i < 3; i++) st.mgrid[i] = i < dims ? mgrid_stride[i] : 1;
  return h;
}

int Runtime::decl_reduction(int size, const char *type, const char *name) {
  OPSB_REQUIRE(inited_, E_STATE, "ops_decl_reduction_handle before ops_init");
  OPSB_REQUIRE(size > 0, E_ARG, "reduction size must be positive");
  Reduction r;
  r.index = (int)reductions_.size();
  r.size = size;
  r.type = type ? type : "double";
  r.elem = type_size_of(r.type.c_str());
  OPSB_REQUIRE(r.elem > 0, E_ARG, "unknown reduction type " + r.type);
  r.name = name ? name : "";
  auto span = [](int bytes) { return (size_t)((std::max(bytes, 64) + 63) / 64 * 64); };
  size_t off = reductions_.empty() ? 0 : (size_t)(reductions_.back().slot_d - red_arena_) + span(reductions_.back().size);
  OPSB_REQUIRE(off + span(size) <= kRedArenaBytes, E_UNSUPPORTED, "reduction handles exceed the 64 KiB arena");
  r.slot_d = red_arena_ + off;
  OPSB_CUDA(cudaMemsetAsync(r.slot_d, 0, span(size), stream_));
  red_dirty_ = true;
  reductions_.push_back(r);
  return r.index;
}

void Runtime::decl_const(const char *name, int dim, const char *type, const void *data) {
  OPSB_REQUIRE(inited_, E_STATE, "ops_decl_const before ops_init");
  execute();  // ops_update_const flushes the queue first (ops_lazy.cpp semantics)
  // "<app>/<name>" updates that app's slot only; a bare name updates every
  // app's slot of that name.
  std::string scope, key;
  split_const_name(name ? name : "", scope, key);
  auto range = registry().consts.equal_range(key);
  int ts = type_size_of(type);
  // Struct-typed constants (CloverLeaf's field_type, for one) have no scalar
  // size: the registered slot size is copied, so a bare name must not match
  // slots of different sizes (2D and 3D field_type, say).
  if (ts <= 0) {
    size_t seen = 0;
    for (auto it = range.first; it != range.second; ++it) {
      if (!scope.empty() && it->second.scope != scope) continue;
      OPSB_REQUIRE(seen == 0 || seen == it->second.bytes, E_ARG,
              "constant '" + key + "' has different layouts in several apps: qualify it as <app>/" + key);
      seen = it->second.bytes;
    }
  }
  bool any = false;
  for (auto it = range.first; it != range.second; ++it) {
    if (!scope.empty() && it->second.scope != scope) continue;
    size_t bytes = ts > 0 ? (size_t)ts * dim : it->second.bytes;
    bytes = std::min(bytes, it->second.bytes);
    OPSB_CUDA(cudaMemcpyToSymbolAsync(it->second.symbol, data, bytes, it->second.offset, cudaMemcpyHostToDevice,
                                      stream_));
    any = true;
  }
  if (any) OPSB_CUDA(cudaStreamSynchronize(stream_));
}

// ---------------------------------------------------------------------------
// Loop enqueue (create_kerneldesc_and_enque, ops/c/src/core/ops_lazy.cpp:1403).
// ---------------------------------------------------------------------------
void Runtime::par_loop(const LoopInfo *loop, const char *name, int blk, int dim, const int *range,
                       const Arg *args, int nargs) {
  OPSB_REQUIRE(inited_, E_STATE, "ops_par_loop before ops_init");
  OPSB_REQUIRE(loop != nullptr, E_NOTFOUND, "unknown loop kernel");
  Block &b = block(blk);
  OPSB_REQUIRE(dim == b.dims, E_ARG, "ops_par_loop dim does not match the block");
  OPSB_REQUIRE(nargs == loop->nparams, E_ARG,
          "loop " + loop->kernel + " takes " + std::to_string(loop->nparams) + " args, got " + std::to_string(nargs));
  OPSB_REQUIRE(nargs <= OPSB_MAX_ARGS, E_ARG, "too many loop args");
  Desc d;
  d.loop = loop;
  d.name = name ? name : loop->kernel;
  d.block = blk;
  d.dim = dim;
  for (int i = 0; i < 3; i++) {
    d.range[2 * i] = i < dim ? range[2 * i] : 0;
    d.range[2 * i + 1] = i < dim ? range[2 * i + 1] : 1;
  }
  d.args.assign(args, args + nargs);
  d.red_first.assign(nargs, 0);
  d.gbl_off.assign(nargs, 0);
  clip_loop(d);  // the rank's slab of the range on a partitioned block
  int nred = 0;
  for (int i = 0; i < nargs; i++) {
    Arg &a = d.args[i];
    const ParamInfo &p = loop->params[i];
    switch (a.kind) {
      case ARG_DAT: {
        Dat &dt = dat(a.dat);
        stencil(a.stencil);
        OPSB_REQUIRE(p.cls == 'A', E_ARG, "loop " + loop->kernel + ": arg " + std::to_string(i) + " is a dat but the kernel expects a pointer");
        OPSB_REQUIRE(p.elem == dt.type_size, E_ARG, "loop " + loop->kernel + ": dat " + dt.name + " element size mismatch");
        OPSB_REQUIRE(dt.dim == 1, E_UNSUPPORTED, "dat " + dt.name + ": multi-component dats are not supported by loop kernels");
        OPSB_REQUIRE(dt.plane < (1LL << 31), E_UNSUPPORTED, "dat " + dt.name + " has a plane of 2^31 elements or more");
        OPSB_REQUIRE(dt.block == blk, E_ARG, "dat " + dt.name + " is declared on another block");
        OPSB_REQUIRE(dt.locked == 0, E_STATE, "dat " + dt.name + " is used in a loop while its raw pointer is held (ops_lib_core.cpp:2321)");
        OPSB_REQUIRE(stencils_[a.stencil].type == 0 || loop->mgrid_ok, E_UNSUPPORTED,
                "loop " + loop->kernel + " is not built for restrict/prolong stencils (mgrid)");
        check_in_allocation(d, a, dt);
        if (a.acc != ACC_READ) dt.host.clear();
        break;
      }
      case ARG_GBL:
        OPSB_REQUIRE(p.cls == 'c' || p.cls == 'p', E_ARG, "loop " + loop->kernel + ": arg " + std::to_string(i) + " is a global but the kernel expects an accessor");
        OPSB_REQUIRE(a.gbl.size() <= 4096, E_ARG, "global argument larger than 4 KiB");
        break;
      case ARG_REDUCE: {
        Reduction &r = reduction(a.red);
        OPSB_REQUIRE(p.cls == 'R', E_ARG, "loop " + loop->kernel + ": reduction arg must bind to a RED<> parameter");
        OPSB_REQUIRE(a.dim <= p.ndim, E_ARG, "reduction " + r.name + " wider than the kernel's accumulator");
        OPSB_REQUIRE(p.elem == r.elem, E_ARG, "reduction " + r.name + " type does not match the kernel parameter");
        OPSB_REQUIRE(a.dim <= OPSB_MAX_RED_DIM && a.dim * r.elem <= r.size, E_ARG, "reduction " + r.name + " too wide");
        OPSB_REQUIRE(nred < OPSB_MAX_REDUCE_ARGS, E_ARG, "too many reductions in one loop");
        OPSB_REQUIRE(a.acc == ACC_INC || a.acc == ACC_MIN || a.acc == ACC_MAX, E_ARG, "reduction access must be INC, MIN or MAX");
        // ops_arg_reduce_core (ops/c/src/core/ops_lib_core.cpp:856): the first use after a result restarts.
        d.red_first[i] = r.initialized ? 0 : 1;
        r.initialized = 1;
        r.acc = a.acc;
        a.elem = r.elem;
        nred++;
        break;
      }
      case ARG_IDX:
        OPSB_REQUIRE(p.cls == 'I', E_ARG, "ops_arg_idx must bind to an IDX parameter");
        break;
      default:
        throw Error(E_ARG, "unknown arg kind");
    }
  }
  exchange_for_loop(d);  // neighbours' rows the loop reads (partitioned blocks)
  LoopRecord rec;
  if (redundant(d, rec)) {
    loops_skipped_++;
    return;
  }
  mark_written(d);
  queue_.push_back(std::move(d));
  qrec_.push_back(std::move(rec));
  loops_enqueued_++;
  if (queue_.size() >= 4096) execute();
}

// Every point a loop argument can touch, the range widened by its stencil's
// offsets along the dimensions the stencil walks, must lie in the dat's
// stored window [lo, hi) (the whole extent [base + d_m, base + d_m + size)
// unless the dat is partitioned across ranks): the reference leaves this to
// the application, a device kernel here would read or write outside its
// buffer. Folded (stride 0) dimensions address index 0.
void Runtime::check_in_allocation(const Desc &d, const Arg &a, const Dat &dt) const {
  const Stencil &st = stencils_[a.stencil];
  for (int k = 0; k < d.dim; k++)
    if (d.range[2 * k + 1] <= d.range[2 * k]) return;  // empty range: nothing is touched
  for (int k = 0; k < d.dim; k++) {
    long long lo, hi;
    if (st.stride[k]) {
      int omin = 0, omax = 0;
      for (int p = 0; p < st.points; p++) {
        int o = st.offs[(size_t)p * st.dims + k];
        if (p == 0 || o < omin) omin = o;
        if (p == 0 || o > omax) omax = o;
      }
      long long x0 = d.range[2 * k], x1 = (long long)d.range[2 * k + 1] - 1;
      if (st.type == 2) {  // restrict: x * stride
        x0 *= st.mgrid[k];
        x1 *= st.mgrid[k];
      } else if (st.type == 1) {  // prolong: floor(x / stride)
        auto fl = [](long long v, long long q) { return v >= 0 ? v / q : -((q - 1 - v) / q); };
        x0 = fl(x0, st.mgrid[k]);
        x1 = fl(x1, st.mgrid[k]);
      }
      lo = x0 + omin;
      hi = x1 + omax;
    } else {
      lo = hi = 0;
    }
    const long long first = dt.lo[k], last = (long long)dt.hi[k] - 1;
    OPSB_REQUIRE(lo >= first && hi <= last, E_ARG,
            "loop " + d.loop->kernel + ": dat " + dt.name + " accessed at [" + std::to_string(lo) + ", " +
                std::to_string(hi) + "] in dimension " + std::to_string(k) + ", allocated [" +
                std::to_string(first) + ", " + std::to_string(last) + "]");
  }
}

// A loop that only reads some dats and writes others is redundant when an
// identical loop (kernel, block, range, args, global values) is already
// queued in this flush and none of its inputs or outputs has been written
// since: running it again would store the same values. (The reference's
// CloverLeaf momentum advection, for one, recomputes its volume and mass
// fluxes for the second velocity component.) Fills `rec` for the new loop.
bool Runtime::redundant(const Desc &d, LoopRecord &rec) {
  const size_t na = d.args.size();
  rec.ver.assign(na, 0);
  rec.pure = fusion_on_ && !d.loop->internal;
  for (size_t i = 0; i < na; i++) {
    const Arg &a = d.args[i];
    if (a.kind == ARG_DAT) {
      if (a.acc != ACC_READ && a.acc != ACC_WRITE) rec.pure = false;
      auto it = dat_ver_.find(a.dat);
      rec.ver[i] = it == dat_ver_.end() ? 0 : it->second;
    } else if (a.kind == ARG_REDUCE || (a.kind == ARG_GBL && a.acc != ACC_READ)) {
      rec.pure = false;
    }
  }
  if (rec.pure) {
    for (size_t q = queue_.size(); q-- > 0;) {
      const LoopRecord &r = qrec_[q];
      const Desc &e = queue_[q];
      if (!r.pure || e.loop != d.loop || e.block != d.block || e.args.size() != na ||
          memcmp(e.range, d.range, sizeof(d.range)) != 0)
        continue;
      bool same = true;
      for (size_t i = 0; i < na && same; i++) {
        const Arg &x = e.args[i], &y = d.args[i];
        same = x.kind == y.kind && x.dat == y.dat && x.stencil == y.stencil && x.acc == y.acc && x.opt == y.opt &&
               x.dim == y.dim && x.gbl == y.gbl && r.ver[i] == rec.ver[i];
      }
      if (same) return true;
    }
  }
  // not redundant: the dats it writes get new versions
  for (size_t i = 0; i < na; i++) {
    const Arg &a = d.args[i];
    if (a.kind == ARG_DAT && a.acc != ACC_READ) {
      const unsigned long long v = ++ver_counter_;
      dat_ver_[a.dat] = v;
      rec.ver[i] = v;
    }
  }
  return false;
}

void Runtime::launch_shape(const int *range, int dim, bool reduces, dim3 &grid, dim3 &block) {
  (void)dim;
  long long nx = std::max(0, range[1] - range[0]);
  long long ny = std::max(0, range[3] - range[2]);
  long long nz = std::max(0, range[5] - range[4]);
  long long nrows = ny * nz;
  int bx = nx >= 128 ? 128 : (nx >= 64 ? 64 : 32);
  int by = 256 / bx;
  long long gx = std::max(1LL, (nx + bx - 1) / bx);
  long long target = 148LL * 16;
  long long gy = std::max(1LL, std::min((nrows + by - 1) / by, std::max(1LL, target / gx)));
  gy = std::min(gy, 65535LL);
  if (reduces) {
    while (gx * gy > kMaxRedBlocks && gy > 1) gy = (gy + 1) / 2;
    if (gx * gy > kMaxRedBlocks) throw Error(E_UNSUPPORTED, "reduction loop too wide");
  }
  grid = dim3((unsigned)gx, (unsigned)gy, 1);
  block = dim3(bx, by, 1);
}

void Runtime::build_params(const Desc &d, LoopParams &lp, int *nred_out) {
  memset(&lp, 0, sizeof(lp));
  for (int i = 0; i < 3; i++) {
    lp.start[i] = d.range[2 * i];
    lp.end[i] = d.range[2 * i + 1];
  }
  lp.ndim = d.dim;
  lp.nargs = (int)d.args.size();
  int nred = 0;
  for (int i = 0; i < lp.nargs; i++) {
    const Arg &a = d.args[i];
    ArgView &v = lp.a[i];
    v.kind = a.kind;
    v.acc = a.acc;
    v.dim = a.dim;
    switch (a.kind) {
      case ARG_DAT: {
        const Dat &dt = *dats_[a.dat];
        const Stencil &st = stencils_[a.stencil];
        // an optional argument keeps its storage pointer, as ops_arg_dat_opt
        // does (ops_lib_core.cpp:1107-1113): kernels test their own flags,
        // which need not agree with the argument's
        v.ptr = dt.origin_ptr();
        v.sx = st.stride[0] ? 1 : 0;
        v.sy = st.stride[1] ? (int)dt.pitch : 0;
        v.sz = st.stride[2] ? (int)dt.plane : 0;
        v.ay = (int)dt.pitch;
        v.az = (int)dt.plane;
        v.mg = st.type;
        for (int k = 0; k < 3; k++) v.ms[k] = st.mgrid[k];
        break;
      }
      case ARG_GBL:
        v.ptr = gbl_dev_ + d.gbl_off[i];
        break;
      case ARG_REDUCE:
        v.ptr = reductions_[a.red].slot_d;
        v.red_index = nred++;
        v.first = d.red_first[i];
        break;
      default:
        break;
    }
  }
  lp.nred = nred;
  lp.red_scratch = red_scratch_;
  lp.red_counter = red_counters_;
  if (nred_out) *nred_out = nred;
}

uint64_t Runtime::queue_key(const std::vector<Desc> &q) const {
  uint64_t h = 0xCBF29CE484222325ULL;
  for (const Desc &d : q) {
    h = mix64(h, (uint64_t)(uintptr_t)d.loop);
    for (int i = 0; i < 6; i++) h = mix64(h, (uint64_t)(uint32_t)d.range[i]);
    for (size_t i = 0; i < d.args.size(); i++) {
      const Arg &a = d.args[i];
      h = mix64(h, ((uint64_t)a.kind << 56) ^ ((uint64_t)a.acc << 48) ^ ((uint64_t)a.opt << 40) ^
                       ((uint64_t)(a.dim & 0xff) << 32) ^ (uint64_t)(uint32_t)a.stencil);
      if (a.kind == ARG_DAT) h = mix64(h, (uint64_t)(uintptr_t)dats_[a.dat]->data_d);
      if (a.kind == ARG_REDUCE) h = mix64(h, ((uint64_t)a.red << 1) | (uint64_t)d.red_first[i]);
      if (a.kind == ARG_GBL) h = mix64(h, (uint64_t)d.gbl_off[i] ^ ((uint64_t)a.gbl.size() << 40));
    }
    // A fused chain resolves a boundary copy loop's field flags when it is
    // planned: the flag values are part of the structure.
    if (const CopyLoopSpec *sp = find_copy_loop(d.loop))
      if (sp->flags_arg >= 0 && sp->flags_arg < (int)d.args.size())
        for (char c : d.args[sp->flags_arg].gbl) h = mix64(h, (uint64_t)(unsigned char)c);
  }
  return h;
}

void Runtime::set_timing(int on) {
  collect_timing();
  timing_on_ = on;
}

double Runtime::alg_bytes(const Desc &d) const {
  double total = 0.0;
  for (const Arg &a : d.args) {
    if (a.kind != ARG_DAT || !a.opt) continue;
    const Dat &dt = *dats_[a.dat];
    const Stencil &st = stencils_[a.stencil];
    double pts = 1.0;
    for (int k = 0; k < d.dim; k++)
      if (st.stride[k]) pts *= std::max(0, d.range[2 * k + 1] - d.range[2 * k]);
    total += pts * dt.elem_size * ((a.acc == ACC_RW || a.acc == ACC_INC) ? 2 : 1);
  }
  return total;
}

void Runtime::timed_launch_begin(const std::string &name, double bytes) {
  if (!timing_on_) return;
  cur_bytes_ = bytes;
  if (event_pool_.empty()) {
    for (int i = 0; i < 64; i++) {
      cudaEvent_t e;
      OPSB_CUDA(cudaEventCreate(&e));
      event_pool_.push_back(e);
    }
  }
  cur_ev_ = event_pool_.back();
  event_pool_.pop_back();
  cur_name_ = name;
  OPSB_CUDA(cudaEventRecord(cur_ev_, stream_));
}

void Runtime::timed_launch_end() {
  if (!timing_on_ || !cur_ev_) return;
  if (event_pool_.empty()) {
    for (int i = 0; i < 64; i++) {
      cudaEvent_t e;
      OPSB_CUDA(cudaEventCreate(&e));
      event_pool_.push_back(e);
    }
  }
  cudaEvent_t e = event_pool_.back();
  event_pool_.pop_back();
  OPSB_CUDA(cudaEventRecord(e, stream_));
  pending_.push_back({cur_name_, cur_ev_, e, cur_bytes_});
  cur_ev_ = nullptr;
  if (pending_.size() > 4096) collect_timing();
}

void Runtime::collect_timing() {
  if (pending_.empty()) return;
  OPSB_CUDA(cudaStreamSynchronize(stream_));
  for (auto &p : pending_) {
    float ms = 0.f;
    OPSB_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
    KTime &k = ktimes_[p.name];
    k.launches++;
    k.ms += ms;
    k.bytes += p.bytes;
    event_pool_.push_back(p.a);
    event_pool_.push_back(p.b);
  }
  pending_.clear();
}

// Every item of a flush, in queue order, with its launch resolved now: fused
// chains (fusion.cpp) and, between them, runtime-internal items, chain rules
// (batched boundary copies) and single loops. Storage moves made by a fused
// chain are visible to the items planned after it only.
void Runtime::plan_items(std::vector<Desc> &q, std::vector<PlanItem> &out, std::vector<int> &renamed,
                         bool &tuning) {
  out.clear();
  renamed.clear();
  tuning = false;
  std::vector<FusedItem> fused;
  plan_fusion(q, fused);
  size_t i = 0;
  for (FusedItem &f : fused) {
    plan_plain(q, i, f.first, out);
    build_fused(q, f);
    if (f.unfused) {
      // the tuner times this chain's loops run one by one: events around them
      tuning = true;
      cudaEvent_t e0 = f.ev0, e1 = f.ev1;
      PlanItem a;
      a.name = "runtime/tune_begin";
      a.run = [e0](cudaStream_t s) { OPSB_CUDA(cudaEventRecord(e0, s)); };
      out.push_back(std::move(a));
      plan_plain(q, f.first, f.first + f.n, out);
      PlanItem b;
      b.name = "runtime/tune_end";
      b.run = [e1](cudaStream_t s) { OPSB_CUDA(cudaEventRecord(e1, s)); };
      out.push_back(std::move(b));
    } else {
      renamed.insert(renamed.end(), f.renamed.begin(), f.renamed.end());
      tuning = tuning || f.tuning;
      PlanItem it;
      it.name = f.name;
      it.bytes = f.bytes;
      it.kernels = 1;
      it.fused_loops = (long long)f.n;
      it.loop_bytes = f.loop_bytes;
      auto launch = f.launch;
      const fuse::FPlan *dplan = f.dplan;
      const int grid = f.grid;
      const size_t smem = (size_t)f.smem;
      cudaEvent_t e0 = f.ev0, e1 = f.ev1;
      it.run = [launch, dplan, grid, smem, e0, e1](cudaStream_t s) {
        if (e0) OPSB_CUDA(cudaEventRecord(e0, s));
        launch(dplan, grid, smem, s);
        OPSB_CUDA(cudaGetLastError());
        if (e1) OPSB_CUDA(cudaEventRecord(e1, s));
      };
      out.push_back(std::move(it));
    }
    i = f.first + f.n;
  }
  plan_plain(q, i, q.size(), out);
}

// The items of q[from, to) that no fused chain covers.
void Runtime::plan_plain(std::vector<Desc> &q, size_t from, size_t to, std::vector<PlanItem> &out) {
  auto &chains = registry().chains;
  size_t i = from;
  while (i < to) {
    if (q[i].loop->internal) {
      out.push_back(q[i].loop->internal == 2 ? prepare_exchange(q[i]) : prepare_swap_outside(q[i]));
      i++;
      continue;
    }
    if (fusion_on_) {
      bool done = false;
      for (auto &rule : chains) {
        int n = rule.match(q, i);
        n = (int)std::min<size_t>((size_t)std::max(n, 0), to - i);
        if (n > 0) {
          out.push_back(rule.prepare(q, i, n));
          i += n;
          done = true;
          break;
        }
      }
      if (done) continue;
      if (lists_on_) {
        const size_t n = list_run(q, i, to);
        if (n >= 2 && prepare_list(q, i, n, out)) {
          i += n;
          continue;
        }
      }
    }
    const Desc &d = q[i];
    LoopParams lp;
    int nred = 0;
    build_params(d, lp, &nred);
    lp.red_counter = red_counters_ + (i % kNumCounters);
    dim3 g, b;
    launch_shape(d.range, d.dim, nred > 0, g, b);
    long long nx = (long long)d.range[1] - d.range[0];
    long long nr = (long long)(d.range[3] - d.range[2]) * (d.range[5] - d.range[4]);
    PlanItem it;
    it.name = d.loop->kernel;
    if ((nx > 0 && nr > 0) || nred > 0) {
      it.bytes = timing_on_ ? alg_bytes(d) : 0.0;
      it.kernels = 1;
      auto launch = d.loop->launch;
      it.run = [lp, g, b, launch](cudaStream_t s) {
        launch(lp, g, b, s);
        OPSB_CUDA(cudaGetLastError());
      };
    }
    out.push_back(std::move(it));
    i++;
  }
}

// Consecutive loops of one kernel that are independent of one another (no
// loop reads or writes a dat another one writes) and carry no reduction: the
// steps of a multi-block application over its blocks, for one. Returns how
// many, from q[i].
size_t Runtime::list_run(const std::vector<Desc> &q, size_t i, size_t to) const {
  const LoopInfo *L = q[i].loop;
  if (L->internal || !L->launch_list) return 0;
  auto eligible = [&](const Desc &d) {
    if (d.loop != L) return false;
    for (int k = 0; k < 3; k++)
      if (d.range[2 * k + 1] <= d.range[2 * k]) return false;
    for (const Arg &a : d.args)
      if (a.kind == ARG_REDUCE) return false;
    return true;
  };
  std::vector<int> written, touched;
  auto has = [](const std::vector<int> &v, int x) { return std::find(v.begin(), v.end(), x) != v.end(); };
  size_t j = i;
  while (j < to && eligible(q[j])) {
    bool ok = true;
    for (const Arg &a : q[j].args)
      if (a.kind == ARG_DAT && (has(written, a.dat) || (a.acc != ACC_READ && has(touched, a.dat)))) ok = false;
    if (!ok) break;
    for (const Arg &a : q[j].args)
      if (a.kind == ARG_DAT) {
        touched.push_back(a.dat);
        if (a.acc != ACC_READ) written.push_back(a.dat);
      }
    j++;
  }
  return j - i;
}

// The work list of q[i, i+n): each loop's parameters and CTA grid (sized as
// launch_shape sizes a single loop's), uploaded now, before any capture, and
// kept by content (a captured graph keeps pointing at them).
bool Runtime::prepare_list(std::vector<Desc> &q, size_t i, size_t n, std::vector<PlanItem> &out) {
  std::vector<LoopParams> lps(n);
  std::vector<ListItem> grids(n);
  int bx = 32;
  for (size_t k = 0; k < n; k++) {
    const int nx = q[i + k].range[1] - q[i + k].range[0];
    bx = std::max(bx, nx >= 128 ? 128 : (nx >= 64 ? 64 : 32));
  }
  const int by = 256 / bx;
  long long total = 0;
  double bytes = 0.0;
  for (size_t k = 0; k < n; k++) {
    const Desc &d = q[i + k];
    int nred = 0;
    build_params(d, lps[k], &nred);
    const long long nx = (long long)d.range[1] - d.range[0];
    const long long nrows = (long long)(d.range[3] - d.range[2]) * (d.range[5] - d.range[4]);
    const long long gx = (nx + bx - 1) / bx;
    long long gy = std::min((nrows + by - 1) / by, std::max(1LL, 148LL * 16 / gx));
    gy = std::max(1LL, std::min(gy, 65535LL));
    grids[k] = {(int)gx, (int)gy, total};
    total += gx * gy;
    if (timing_on_) bytes += alg_bytes(d);
  }
  if (total > 0x7fffffffLL) return false;
  const size_t pb = n * sizeof(LoopParams), gb = n * sizeof(ListItem);
  uint64_t h = 0xCBF29CE484222325ULL;
  for (const unsigned char *c = (const unsigned char *)lps.data(), *e = c + pb; c < e; c++) h = (h ^ *c) * 0x100000001B3ULL;
  for (const unsigned char *c = (const unsigned char *)grids.data(), *e = c + gb; c < e; c++)
    h = (h ^ *c) * 0x100000001B3ULL;
  h ^= n;
  char *dev = nullptr;
  auto it = list_cache_.find(h);
  if (it != list_cache_.end()) {
    dev = it->second;
  } else {
    OPSB_CUDA(cudaMalloc(&dev, pb + gb));
    OPSB_CUDA(cudaMemcpyAsync(dev, lps.data(), pb, cudaMemcpyHostToDevice, stream_));
    OPSB_CUDA(cudaMemcpyAsync(dev + pb, grids.data(), gb, cudaMemcpyHostToDevice, stream_));
    list_cache_[h] = dev;
  }
  PlanItem p;
  p.name = q[i].loop->kernel;
  p.kernels = 1;
  p.bytes = bytes;
  auto launch = q[i].loop->launch_list;
  const LoopParams *dl = reinterpret_cast<const LoopParams *>(dev);
  const ListItem *dg = reinterpret_cast<const ListItem *>(dev + pb);
  const int cnt = (int)n;
  const dim3 block(bx, by, 1);
  p.run = [launch, dl, dg, cnt, total, block](cudaStream_t s) {
    launch(dl, dg, cnt, total, block, s);
    OPSB_CUDA(cudaGetLastError());
  };
  out.push_back(std::move(p));
  list_loops_ += (long long)n;
  list_launches_++;
  return true;
}

void Runtime::launch_plan(std::vector<PlanItem> &items) {
  for (PlanItem &it : items) {
    if (!it.run) continue;
    timed_launch_begin(it.name, it.bytes);
    it.run(stream_);
    timed_launch_end();
    kernels_launched_ += it.kernels;
    if (it.fused_loops > 0) {
      fstats_.chains++;
      fstats_.loops += it.fused_loops;
      fstats_.bytes += it.bytes;
      fstats_.loop_bytes += it.loop_bytes;
    }
  }
}

// A captured flush replayed: the dats its fused chains renamed move again.
void Runtime::apply_renames(const std::vector<int> &renamed) {
  for (int di : renamed) {
    Dat &d = *dats_[di];
    std::swap(d.data_d, shadow_.at(di));
    d.host.clear();
  }
}

void Runtime::add_fusion_stats(const FusionStats &s) {
  fstats_.chains += s.chains;
  fstats_.loops += s.loops;
  fstats_.bytes += s.bytes;
  fstats_.loop_bytes += s.loop_bytes;
}

void Runtime::run_queue(std::vector<Desc> &q) {
  red_dirty_ = true;
  elide_copies(q);
  // OPSB_TRACE_QUEUE=1: every flushed loop to stderr (kernel, range, per dat
  // arg: name, access, stencil points), for analysing loop chains
  static const bool trace = getenv("OPSB_TRACE_QUEUE") != nullptr;
  if (trace) {
    fprintf(stderr, "flush %zu loops\n", q.size());
    for (const Desc &d : q) {
      fprintf(stderr, "  %s [%d,%d)x[%d,%d)", d.loop->kernel.c_str(), d.range[0], d.range[1], d.range[2], d.range[3]);
      for (const Arg &a : d.args)
        if (a.kind == ARG_DAT)
          fprintf(stderr, " %s:%c%d", dat(a.dat).name.c_str(), "WRIMXX"[a.acc == ACC_READ ? 2 : a.acc == ACC_WRITE ? 0 : a.acc == ACC_RW ? 1 : 3],
                  stencils_[a.stencil].points);
      fprintf(stderr, "\n");
    }
  }
  // Stage the READ globals of the whole flush into the device arena.
  gbl_used_ = 0;
  for (Desc &d : q) {
    for (size_t i = 0; i < d.args.size(); i++) {
      const Arg &a = d.args[i];
      if (a.kind != ARG_GBL) continue;
      size_t off = (gbl_used_ + 15) & ~(size_t)15;
      OPSB_REQUIRE(off + a.gbl.size() <= gbl_cap_, E_UNSUPPORTED, "global argument arena exhausted in one flush");
      memcpy(gbl_host_.data() + off, a.gbl.data(), a.gbl.size());
      d.gbl_off[i] = off;
      gbl_used_ = off + a.gbl.size();
    }
  }
  if (gbl_used_ > 0)
    OPSB_CUDA(cudaMemcpyAsync(gbl_dev_, gbl_host_.data(), gbl_used_, cudaMemcpyHostToDevice, stream_));

  const bool use_graphs = graphs_on_ && !timing_on_ && q.size() >= 2;
  GraphEntry *ge = nullptr;
  if (use_graphs) {
    ge = &graphs_[queue_key(q)];
    if (ge->exec) {
      OPSB_CUDA(cudaGraphLaunch(ge->exec, stream_));
      graphs_launched_++;
      kernels_launched_ += ge->kernels;
      apply_renames(ge->renamed);
      add_fusion_stats(ge->fstats);
      return;
    }
  }
  std::vector<PlanItem> items;
  std::vector<int> renamed;
  bool tuning = false;
  plan_items(q, items, renamed, tuning);
  if (!use_graphs || tuning) {
    launch_plan(items);
    return;
  }
  ge->seen++;
  if (ge->seen < 2) {
    launch_plan(items);
    return;
  }
  // Second sighting of this queue structure: capture it once, replay from now on.
  cudaGraph_t graph = nullptr;
  const long long before = kernels_launched_;
  const FusionStats fs0 = fstats_;
  OPSB_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
  try {
    launch_plan(items);
  } catch (...) {
    cudaStreamEndCapture(stream_, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  OPSB_CUDA(cudaStreamEndCapture(stream_, &graph));
  ge->kernels = kernels_launched_ - before;
  kernels_launched_ = before;
  ge->renamed = renamed;
  ge->fstats.chains = fstats_.chains - fs0.chains;
  ge->fstats.loops = fstats_.loops - fs0.loops;
  ge->fstats.bytes = fstats_.bytes - fs0.bytes;
  ge->fstats.loop_bytes = fstats_.loop_bytes - fs0.loop_bytes;
  fstats_ = fs0;
  OPSB_CUDA(cudaGraphInstantiate(&ge->exec, graph, 0));
  cudaGraphDestroy(graph);
  OPSB_CUDA(cudaGraphLaunch(ge->exec, stream_));
  graphs_launched_++;
  kernels_launched_ += ge->kernels;
  add_fusion_stats(ge->fstats);
}

void Runtime::execute() {
  if (!inited_ || queue_.empty()) return;
  std::vector<Desc> q;
  q.swap(queue_);
  qrec_.clear();
  dat_ver_.clear();
  run_queue(q);
}

void Runtime::reduction_result(int handle, void *out) {
  Reduction &r = reduction(handle);
  execute();
  if (red_dirty_) {
    const Reduction &last = reductions_.back();
    const size_t used = (size_t)(last.slot_d - red_arena_) + (size_t)last.size;
    OPSB_CUDA(cudaMemcpyAsync(red_host_, red_arena_, used, cudaMemcpyDeviceToHost, stream_));
    OPSB_CUDA(cudaStreamSynchronize(stream_));
    red_dirty_ = false;
  }
  memcpy(out, red_host_ + (r.slot_d - red_arena_), r.size);
  if (partitioned_ && nranks() > 1) combine_reduction(r, out);
  r.initialized = 0;  // ops_reduction_result_char resets the handle (ops_lib_core.cpp:1143)
}

// ---------------------------------------------------------------------------
// Data access. A partitioned dat's data are its owned part (the extents
// ops_dat_get_extents reports, as the reference's MPI backend does,
// ops/c/src/mpi/ops_mpi_rt_support.cpp:2216-2225); otherwise the whole dat.
// ---------------------------------------------------------------------------
namespace {
// The stored x rows (pitch elements each, in storage order) that hold a
// dat's owned part: the first one and how many.
void owned_rows(const Dat &d, size_t *first, size_t *n) {
  const size_t ny = (size_t)(d.hi[1] - d.lo[1]), nz = (size_t)(d.hi[2] - d.lo[2]);
  if (d.split == 2) {
    *first = (size_t)(d.own_lo[2] - d.lo[2]) * ny;
    *n = (size_t)(d.own_hi[2] - d.own_lo[2]) * ny;
  } else if (d.split == 1) {  // 2D blocks: nz == 1
    *first = (size_t)(d.own_lo[1] - d.lo[1]);
    *n = (size_t)(d.own_hi[1] - d.own_lo[1]) * nz;
  } else {
    *first = 0;
    *n = ny * nz;
  }
}
}  // namespace

size_t Runtime::dat_data_bytes(int di) {
  Dat &d = dat(di);
  size_t first, n;
  owned_rows(d, &first, &n);
  return (size_t)d.size[0] * d.elem_size * n;
}

void Runtime::dat_set_data(int di, const void *host, size_t bytes) {
  execute();
  Dat &d = dat(di);
  OPSB_REQUIRE(d.locked == 0, E_STATE, "ops_dat_set_data on a dat whose raw pointer is held");
  size_t row = (size_t)d.size[0] * d.elem_size;
  size_t first, rows;
  owned_rows(d, &first, &rows);
  OPSB_REQUIRE(bytes == row * rows, E_ARG, "ops_dat_set_data: buffer size does not match the dat extent");
  OPSB_CUDA(cudaMemcpy2DAsync(d.data_d + ((size_t)d.pad_front + first * d.pitch) * d.elem_size,
                              (size_t)d.pitch * d.elem_size, host, row, row, rows, cudaMemcpyHostToDevice, stream_));
  OPSB_CUDA(cudaStreamSynchronize(stream_));
  d.host.clear();
  if (d.split >= 0) d.valid = 0;  // the neighbours' copies of the owned rows are stale
}

void Runtime::dat_fetch_data(int di, void *host, size_t bytes) {
  execute();
  Dat &d = dat(di);
  size_t row = (size_t)d.size[0] * d.elem_size;
  size_t first, rows;
  owned_rows(d, &first, &rows);
  OPSB_REQUIRE(bytes == row * rows, E_ARG, "ops_dat_fetch_data: buffer size does not match the dat extent");
  OPSB_CUDA(cudaMemcpy2DAsync(host, row, d.data_d + ((size_t)d.pad_front + first * d.pitch) * d.elem_size,
                              (size_t)d.pitch * d.elem_size, row, rows, cudaMemcpyDeviceToHost, stream_));
  OPSB_CUDA(cudaStreamSynchronize(stream_));
}

void Runtime::dat_get_extents(int di, int *disp, int *size) {
  Dat &d = dat(di);
  int nd = blocks_[d.block].dims;
  for (int i = 0; i < nd; i++) {
    if (disp) disp[i] = d.own_lo[i] - (d.base[i] + d.d_m[i]);
    if (size) size[i] = d.own_hi[i] - d.own_lo[i];
  }
}

// memspace: 1 = host, 2 = device (ops_memspace, ops/c/include/ops_lib_core.h).
char *Runtime::dat_get_raw_pointer(int di, int memspace, int *stride_elems) {
  execute();
  Dat &d = dat(di);
  OPSB_REQUIRE(d.locked == 0, E_STATE, "raw pointer already held for dat " + d.name);
  if (stride_elems) {
    stride_elems[0] = (int)d.pitch;
    stride_elems[1] = d.hi[1] - d.lo[1];
    stride_elems[2] = d.hi[2] - d.lo[2];
  }
  if (memspace == 2) {
    OPSB_CUDA(cudaStreamSynchronize(stream_));
    d.locked = 2;
    return d.origin_ptr();
  }
  d.host.resize(d.bytes);
  OPSB_CUDA(cudaMemcpyAsync(d.host.data(), d.data_d, d.bytes, cudaMemcpyDeviceToHost, stream_));
  OPSB_CUDA(cudaStreamSynchronize(stream_));
  d.locked = 1;
  return d.host.data() + d.origin * d.elem_size;
}

void Runtime::dat_release_raw_data(int di, int acc) {
  Dat &d = dat(di);
  OPSB_REQUIRE(d.locked != 0, E_STATE, "ops_dat_release_raw_data without a matching ops_dat_get_raw_pointer");
  if (d.locked == 1 && acc != ACC_READ) {
    OPSB_CUDA(cudaMemcpyAsync(d.data_d, d.host.data(), d.bytes, cudaMemcpyHostToDevice, stream_));
    OPSB_CUDA(cudaStreamSynchronize(stream_));
  }
  if (acc != ACC_READ && d.split >= 0) d.valid = 0;
  d.locked = 0;
}

void Runtime::release_to(const Mark &m) {
  execute();
  OPSB_CUDA(cudaStreamSynchronize(stream_));
  // Cached graphs may reference storage about to be freed.
  for (auto &kv : graphs_)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  graphs_.clear();
  while (dats_.size() > m.dats) {
    const int di = (int)dats_.size() - 1;
    if (dats_.back() && dats_.back()->data_d) recycle_dat_storage(dats_.back()->data_d, dats_.back()->bytes);
    auto sh = shadow_.find(di);
    if (sh != shadow_.end()) {
      if (sh->second) recycle_dat_storage(sh->second, dats_.back()->bytes);
      shadow_.erase(sh);
    }
    dats_.pop_back();
  }
  release_fusion_plans();
  if (slabs_.size() > m.blocks) slabs_.resize(m.blocks);
  partitioned_ = !slabs_.empty();
  while (reductions_.size() > m.reductions) {
    reductions_.pop_back();
  }
  stencils_.resize(std::min(stencils_.size(), m.stencils));
  blocks_.resize(std::min(blocks_.size(), m.blocks));
}

// Storage for a new dat: a kept block of exactly this size if there is one,
// else a new allocation. When the device is out of memory the kept blocks
// (which no other allocator in the process can use) are freed and the
// allocation is tried once more.
char *Runtime::alloc_dat_storage(size_t bytes) {
  const size_t n = bytes > 0 ? bytes : 256;
  auto it = spare_.find(n);
  if (it != spare_.end()) {
    char *p = it->second;
    spare_.erase(it);
    spare_bytes_ -= n;
    return p;
  }
  char *p = nullptr;
  cudaError_t e = cudaMalloc(&p, n);
  if (e == cudaErrorMemoryAllocation && !spare_.empty()) {
    cudaGetLastError();  // clear the (non-sticky) allocation error
    release_spare_storage();
    p = nullptr;
    e = cudaMalloc(&p, n);
  }
  cuda_check(e, "cudaMalloc of dat storage");
  return p;
}

size_t Runtime::release_spare_storage() {
  if (spare_.empty()) return 0;
  if (stream_) OPSB_CUDA(cudaStreamSynchronize(stream_));
  size_t freed = 0;
  for (auto &kv : spare_) {
    cudaFree(kv.second);
    freed += kv.first;
  }
  spare_.clear();
  spare_bytes_ = 0;
  return freed;
}

void Runtime::discard_queue() {
  queue_.clear();
  qrec_.clear();
  dat_ver_.clear();
}

// Called with the stream idle (release_to synchronizes first).
void Runtime::recycle_dat_storage(char *p, size_t bytes) {
  const size_t n = bytes > 0 ? bytes : 256;
  if (spare_bytes_ + n > kSpareCap) {
    cudaFree(p);
    return;
  }
  spare_.emplace(n, p);
  spare_bytes_ += n;
}

void Runtime::dat_swap(int a, int b) {
  execute();
  Dat &x = dat(a);
  Dat &y = dat(b);
  OPSB_REQUIRE(x.bytes == y.bytes && x.pitch == y.pitch && x.origin == y.origin && x.elem_size == y.elem_size, E_ARG,
          "dat_swap needs two dats of identical layout");
  std::swap(x.data_d, y.data_d);
  x.host.clear();
  y.host.clear();
}

}  // namespace opsb
