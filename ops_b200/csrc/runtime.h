// OPS-B200 host runtime: declarations, device data, lazy loop queue,
// reductions, constants and the launch of registered loop kernels.
//
// Semantics follow the reference runtime:
//   dats            ops/c/src/core/ops_lib_core.cpp:445-548 (metadata),
//                   ops/c/src/core/ops_device_singlenode_common.cpp:44-107
//   stencils        ops/c/src/core/ops_lib_core.cpp:640-832
//   args            ops/c/src/core/ops_lib_core.cpp:856,1047-1118
//   lazy queue      ops/c/src/core/ops_lazy.cpp:186-275 (enqueue),
//                   :1248-1377 (ops_execute), :1403-1440 (descriptor + hash)
//   reductions      ops/c/src/core/ops_lib_core.cpp:1119-1143
//   raw data access ops/c/src/core/ops_dummy_singlenode.cpp:662-850
// The B200 design differs where the hardware asks for it: dat rows are
// pitched to 128 bytes in HBM, reductions finish on the device and stay
// there until a result is requested, a flushed queue is replayed as a CUDA
// graph once its structure repeats, and registered chain kernels replace
// runs of queued loops they cover exactly (fusion).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <functional>
#include <initializer_list>
#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "decomp.h"
#include "ops_b200_device.cuh"

namespace opsb {
namespace fuse {
struct FPlan;
}
class FusionPlanner;
struct FusionState;

// Error codes of the C-ABI (include/ops_b200.h).
enum ErrCode { E_OK = 0, E_ARG = -1, E_CUDA = -2, E_STATE = -3, E_NOTFOUND = -4, E_TIMEOUT = -5, E_UNSUPPORTED = -6 };

struct Error {
  int code;
  std::string msg;
  Error(int c, std::string m) : code(c), msg(std::move(m)) {}
};

void cuda_check(cudaError_t e, const char *what);
#define OPSB_CUDA(call) ::opsb::cuda_check((call), #call)

struct Block {
  int index = 0, dims = 0;
  std::string name;
};

struct Dat {
  int index = 0, block = 0, dim = 1, type_size = 8, elem_size = 8;
  int size[3] = {1, 1, 1};  // extent including halos (ops_dat_core::size)
  int base[3] = {0, 0, 0}, d_m[3] = {0, 0, 0}, d_p[3] = {0, 0, 0};
  int pad_front = 0;        // elements before logical column d_m[0]
  long long pitch = 0;      // elements per x row (>= size[0] + pad_front)
  long long plane = 0;      // elements per xy plane
  long long origin = 0;     // element offset of logical index (0,0,0)
  char *data_d = nullptr;   // device allocation
  size_t bytes = 0;
  std::string type, name;
  int locked = 0;           // 0 free, 1 host raw pointer out, 2 device raw pointer out
  std::vector<char> host;   // host mirror for host raw pointers
  // The stored window [lo, hi) and the owned part [own_lo, own_hi) of each
  // dimension, in logical indices: the whole extent [base + d_m, base + d_m
  // + size) unless the dat is partitioned across ranks (decomp.h), when the
  // split dimension keeps the rank's slab plus its neighbours' halo rows.
  int lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  int own_lo[3] = {0, 0, 0}, own_hi[3] = {1, 1, 1};
  int split = -1;           // dimension split across ranks (-1: whole)
  int valid = 0;            // halo rows holding the neighbours' current values
  char *origin_ptr() const { return data_d + origin * elem_size; }
};

struct Stencil {
  int index = 0, dims = 0, points = 0;
  std::vector<int> offs;   // points*dims
  int stride[3] = {1, 1, 1};
  int type = 0;            // 0 plain, 1 prolong, 2 restrict (ops_stencil_core::type)
  int mgrid[3] = {1, 1, 1};  // ops_stencil_core::mgrid_stride
  std::string name;
};

struct Reduction {
  int index = 0, size = 0;  // size in bytes
  int elem = 8;
  std::string type, name;
  char *slot_d = nullptr;   // device slot holding the running value
  int initialized = 0;      // ops_reduction_core::initialized
  int acc = -1;
};

// A loop argument as the host sees it (ops_arg, ops/c/include/ops_lib_core.h:509).
struct Arg {
  int kind = ARG_DAT;
  int dat = -1, stencil = -1, dim = 1, acc = ACC_READ, opt = 1, red = -1;
  int elem = 8;             // GBL/REDUCE element size in bytes
  std::vector<char> gbl;    // GBL payload, copied at enqueue like ops_lazy.cpp:1434-1438
};

struct LoopInfo {
  std::string kernel;       // registered name
  int nparams = 0;
  ParamInfo params[OPSB_MAX_ARGS];
  int ndim = 2;             // accessor dimensionality (0 when the kernel has none)
  int copy_dst = -1, copy_src = -1;  // pure copy kernels: which args are dst/src
  int internal = 0;         // runtime-internal item (not launched through exec_loop)
  int mgrid_ok = 0;         // the kernel maps multigrid (restrict/prolong) stencils
  void (*launch)(const LoopParams &, dim3, dim3, cudaStream_t) = nullptr;
  // several loops of this kernel in one launch (exec_loop_list); null for
  // kernels with their own launch
  void (*launch_list)(const LoopParams *, const ListItem *, int, long long, dim3, cudaStream_t) = nullptr;
};

// A queued loop (ops_kernel_descriptor, ops/c/include/ops_internal2.h:141-157).
struct Desc {
  const LoopInfo *loop = nullptr;
  std::string name;
  int block = 0, dim = 2;
  int range[6] = {0, 1, 0, 1, 0, 1};
  std::vector<Arg> args;
  std::vector<int> red_first;  // per arg: 1 if the reduction handle restarts here
  std::vector<size_t> gbl_off; // per arg: offset of its GBL payload in the arena
  uint64_t hash = 0;
};

// A launch prepared when a flush is planned: the device work of one queued
// loop, or of a run of loops that a chain rule or the fuser replaces, with
// every storage address it uses resolved at planning time (a fused chain can
// move a dat's storage; the loops after it see the new storage, the loops
// before it the old). Planning happens before any graph capture, so `run`
// only launches.
struct PlanItem {
  std::string name;           // timing name (loop kernel, rule or fused group)
  double bytes = 0.0;         // compulsory bytes (per-kernel timing)
  long long kernels = 0;      // kernels `run` launches
  long long fused_loops = 0;  // fused chain: loops it covers
  double loop_bytes = 0.0;    // fused chain: the covered loops' own compulsory bytes
  std::function<void(cudaStream_t)> run;
};

// A replacement for a run of queued loops. `match` inspects the queue from
// position i and returns how many descriptors it covers (0 = no match);
// `prepare` resolves the replacement's launches at planning time.
struct ChainRule {
  std::string name;
  std::function<int(const std::vector<Desc> &, size_t)> match;
  std::function<PlanItem(const std::vector<Desc> &, size_t, int)> prepare;
};

// A run of queued loops that the fuser (fusion.cpp) executes as one kernel.
struct FusedItem {
  size_t first = 0, n = 0;
  std::string name;
  double bytes = 0.0, loop_bytes = 0.0;  // compulsory bytes fused / as separate loops
  bool tuning = false;                   // this execution times a candidate tile shape
  bool unfused = false;                  // the candidate is the loops run one by one
  uint64_t key = 0;
  int shape = 0, grid = 0, smem = 0;
  std::vector<int> renamed;              // dats moved to their shadow storage by this chain
  void (*launch)(const fuse::FPlan *, int, size_t, cudaStream_t) = nullptr;
  fuse::FPlan *dplan = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::shared_ptr<void> analysis;        // the planner's analysis until the plan is built
};

struct LoopStats {
  long long count = 0;
};

// A loop kernel whose every point only copies, for each listed argument f,
//   if (flags == nullptr || flags[flag[f]] == 1) a_f(0,0,0) = (neg ? -1 : 1) * a_f(off)
// with `flags` the int array of global argument `flags_arg` (-1: no flags).
// Runs of such loops are executed as batches of independent copies
// (copy_batch.cu) instead of one launch each.
struct CopyLoopSpec {
  int nfields = 0;
  int arg[8] = {0}, flag[8] = {0};
  int flags_arg = -1;
  int neg = 0;
  int off[3] = {0, 0, 0};
};
void register_copy_loop(const std::string &kernel, const CopyLoopSpec &spec);
const CopyLoopSpec *find_copy_loop(const LoopInfo *loop);

class Runtime {
 public:
  static Runtime &get();
  static bool exists();
  static void destroy();

  void init(int device, int diags);
  bool initialized() const { return inited_; }

  int decl_block(int dims, const char *name);
  int decl_dat(int block, int dim, const int *size, const int *base, const int *d_m, const int *d_p,
               const void *data, int type_size, const char *type, const char *name);
  int decl_stencil(int dims, int points, const int *offs, const int *stride, const char *name);
  // ops_decl_restrict_stencil (type 2) / ops_decl_prolong_stencil (type 1)
  // (ops/c/src/core/ops_lib_core.cpp:740-833)
  int decl_mgrid_stencil(int dims, int points, const int *offs, const int *mgrid_stride, int type, const char *name);
  int decl_reduction(int size, const char *type, const char *name);
  // ops_decl_halo / ops_decl_halo_group / ops_halo_transfer
  // (ops/c/src/core/ops_lib_core.cpp:998-1040, ops_device_singlenode_common.cpp:262-346)
  int decl_halo(int from, int to, const int *iter, const int *from_base, const int *to_base, const int *from_dir,
                const int *to_dir);
  int decl_halo_group(int n, const int *halos);
  void halo_transfer(int group);
  void decl_const(const char *name, int dim, const char *type, const void *data);

  void par_loop(const LoopInfo *loop, const char *name, int block, int dim, const int *range,
                const Arg *args, int nargs);
  void execute();
  void reduction_result(int handle, void *out);

  // Data access (ops_dat_* in ops/c/src/core/ops_dummy_singlenode.cpp:611-850).
  void dat_set_data(int dat, const void *host, size_t bytes);
  void dat_fetch_data(int dat, void *host, size_t bytes);
  void dat_get_extents(int dat, int *disp, int *size);
  size_t dat_data_bytes(int dat);  // bytes of dat_set_data / dat_fetch_data
  char *dat_get_raw_pointer(int dat, int memspace, int *stride_elems);
  void dat_release_raw_data(int dat, int acc);
  void dat_swap(int a, int b);  // exchange device storage of two same-shape dats

  Dat &dat(int i);
  Stencil &stencil(int i);
  Reduction &reduction(int i);
  Block &block(int i);
  int ndats() const { return (int)dats_.size(); }
  cudaStream_t stream() const { return stream_; }

  // Registry of loops (by kernel name) and of named device constants.
  static void register_loop(const LoopInfo &info);
  static const LoopInfo *find_loop(const std::string &kernel);
  // A named constant (ops_decl_const / ops_update_const) maps to `bytes` at
  // `offset` inside a __constant__ symbol; one name may feed several modules.
  static void register_const(const std::string &name, const void *symbol, size_t offset, size_t bytes);
  static void register_chain(const ChainRule &rule);

  // Build the device-side view of a queued loop.
  void build_params(const Desc &d, LoopParams &lp, int *nred_out);
  static void launch_shape(const int *range, int dim, bool reduces, dim3 &grid, dim3 &block);

  // Counters.
  long long kernels_launched() const { return kernels_launched_; }
  long long graphs_launched() const { return graphs_launched_; }
  long long loops_enqueued() const { return loops_enqueued_; }
  void count_kernels(long long n) { kernels_launched_ += n; }
  void set_graphs(int on) { graphs_on_ = on; }
  // Per-kernel CUDA-event timing (launches are bracketed by events on the
  // runtime stream; graphs are bypassed while it is on).
  void set_timing(int on);
  void collect_timing();
  struct KTime { long long launches = 0; double ms = 0.0; double bytes = 0.0; };
  const std::map<std::string, KTime> &kernel_times() { collect_timing(); return ktimes_; }
  void clear_timing() { collect_timing(); ktimes_.clear(); }
  void timed_launch_begin(const std::string &name, double alg_bytes = 0.0);
  // Compulsory bytes of one loop: each dat arg's points once, RW/INC twice.
  double alg_bytes(const Desc &d) const;
  void timed_launch_end();
  void set_fusion(int on) { fusion_on_ = on; }
  void set_tiling(int on) { tiling_on_ = on; }
  void set_lists(int on) { lists_on_ = on; }
  void set_tile_candidate(int c);
  long long list_plans() const { return list_launches_; }
  long long list_loops() const { return list_loops_; }
  long long loops_skipped() const { return loops_skipped_; }
  int fusion_enabled() const { return fusion_on_; }
  int diags() const { return diags_; }
  void reset_counters() { kernels_launched_ = graphs_launched_ = loops_enqueued_ = 0; }
  char *red_scratch() const { return red_scratch_; }
  char *gbl_device() const { return gbl_dev_; }  // this flush's staged globals (Desc::gbl_off)
  unsigned int *red_counters() const { return red_counters_; }
  static constexpr int kMaxRedBlocks = 65536;
  static constexpr int kNumCounters = 256;
  static constexpr size_t kRedArenaBytes = 1 << 16;

  // Declarations made by one app call are released when it returns.
  struct Mark { size_t blocks, dats, stencils, reductions; };
  Mark mark() const { return {blocks_.size(), dats_.size(), stencils_.size(), reductions_.size()}; }
  void release_to(const Mark &m);
  // Drops the queued loops without running them (an app driver's error
  // path, before it releases its declarations).
  void discard_queue();
  // Frees the dat storage kept for reuse (see alloc_dat_storage); returns
  // the bytes given back.
  size_t release_spare_storage();
  size_t spare_storage_bytes() const { return spare_bytes_; }

  ~Runtime();

  // Loop-chain fusion statistics since the last reset: fused kernels
  // launched, loops they covered, and their compulsory bytes fused and as
  // separate loops.
  struct FusionStats { long long chains = 0, loops = 0; double bytes = 0.0, loop_bytes = 0.0; };
  const FusionStats &fusion_stats() const { return fstats_; }
  void reset_fusion_stats() { fstats_ = FusionStats(); }

  // Decomposition across processes (decomp.cpp). The transport is set
  // before ops_partition; without one (or with one rank) partition is a
  // no-op, as ops_partition is in the reference's single-process backends.
  void set_transport(std::unique_ptr<Transport> t);
  void partition(const char *routine);
  int nranks() const;
  int rank() const;
  bool partitioned() const { return partitioned_; }
  const Slab &slab(int block) const;
  long long exchanges() const { return exchanges_; }
  Transport *transport() const { return transport_.get(); }
  int device() const { return device_; }

 private:
  friend class FusionPlanner;
  Runtime() = default;
  void run_queue(std::vector<Desc> &q);
  void elide_copies(std::vector<Desc> &q);
  PlanItem prepare_swap_outside(const Desc &d);
  PlanItem prepare_exchange(const Desc &d);
  void window_dat(Dat &d);
  void clip_loop(Desc &d);
  void exchange_for_loop(const Desc &d);
  void mark_written(const Desc &d);
  void exchange_dats(const std::vector<int> &dats);
  void combine_reduction(const Reduction &r, void *value);
  void plan_items(std::vector<Desc> &q, std::vector<PlanItem> &out, std::vector<int> &renamed, bool &tuning);
  void launch_plan(std::vector<PlanItem> &items);
  void plan_plain(std::vector<Desc> &q, size_t from, size_t to, std::vector<PlanItem> &out);
  size_t list_run(const std::vector<Desc> &q, size_t i, size_t to) const;
  bool prepare_list(std::vector<Desc> &q, size_t i, size_t n, std::vector<PlanItem> &out);
  void plan_fusion(const std::vector<Desc> &q, std::vector<FusedItem> &items);
  void build_fused(const std::vector<Desc> &q, FusedItem &item);
  FusionState &fusion_state();
  void release_fusion_state();
  void release_fusion_plans();
  void apply_renames(const std::vector<int> &renamed);
  void add_fusion_stats(const FusionStats &s);
  uint64_t queue_key(const std::vector<Desc> &q) const;

  bool inited_ = false;
  int device_ = 0, diags_ = 0;
  cudaStream_t stream_ = nullptr;
  std::vector<Block> blocks_;
  std::vector<std::unique_ptr<Dat>> dats_;
  // Dat storage given back by release_to (an app driver's teardown), kept
  // by size for the next dats of the same size instead of cudaFree /
  // cudaMalloc of gigabytes per app call; at most kSpareCap bytes are kept.
  static constexpr size_t kSpareCap = (size_t)64 << 30;
  std::multimap<size_t, char *> spare_;
  size_t spare_bytes_ = 0;
  char *alloc_dat_storage(size_t bytes);
  void recycle_dat_storage(char *p, size_t bytes);
  struct Halo {
    int from = -1, to = -1;
    int iter[3], fbase[3], tbase[3], fdir[3], tdir[3];
  };
  std::vector<Halo> halos_;
  std::vector<std::vector<int>> halo_groups_;
  void *halo_desc_d_ = nullptr;
  size_t halo_desc_cap_ = 0;
  std::vector<Stencil> stencils_;
  std::vector<Reduction> reductions_;
  std::vector<Desc> queue_;

  // GBL arena: host staging and its device copy, refilled per flush.
  std::vector<char> gbl_host_;
  char *gbl_dev_ = nullptr;
  size_t gbl_cap_ = 0;
  size_t gbl_used_ = 0;

  char *red_scratch_ = nullptr;
  unsigned int *red_counters_ = nullptr;
  // Reduction handles live in one device arena; a result request copies the
  // whole arena once to pinned memory and serves further requests from
  // there until loops run again.
  char *red_arena_ = nullptr;
  char *red_host_ = nullptr;
  bool red_dirty_ = true;

  struct GraphEntry {
    int seen = 0;
    cudaGraphExec_t exec = nullptr;
    long long kernels = 0;
    std::vector<int> renamed;  // storage moves the captured flush makes (replayed on the host)
    FusionStats fstats;        // fusion statistics of one replay
  };
  // Fused chains write renamed dats into a shadow allocation of the same
  // size, which then becomes the dat's storage (the old one the shadow).
  std::unordered_map<int, char *> shadow_;
  FusionState *fusion_state_ = nullptr;  // owned; created and freed in fusion.cpp
  FusionStats fstats_;
  std::unordered_map<uint64_t, GraphEntry> graphs_;
  int graphs_on_ = 1;
  int timing_on_ = 0;
  struct PendingTime { std::string name; cudaEvent_t a, b; double bytes; };
  std::vector<PendingTime> pending_;
  std::vector<cudaEvent_t> event_pool_;
  std::map<std::string, KTime> ktimes_;
  std::string cur_name_;
  double cur_bytes_ = 0.0;
  cudaEvent_t cur_ev_ = nullptr;
  int fusion_on_ = 1;
  int tiling_on_ = 1;  // loop-chain fusion into tiled kernels (needs fusion_on_)
  int lists_on_ = 1;   // runs of one kernel over several blocks in one launch (needs fusion_on_)
  int tile_candidate_ = -1;  // >= 0: every fused chain runs this tuning candidate (no tuning)
  // Redundant-loop elimination within one flush: per queued loop, the
  // version of each dat arg (read: as observed, written: as produced);
  // dat versions count the writes of the queued loops and restart at every
  // flush (every other way of changing a dat flushes first).
  struct LoopRecord {
    bool pure = false;                 // only READ/WRITE dats, READ globals, indices
    std::vector<unsigned long long> ver;
  };
  std::vector<LoopRecord> qrec_;
  std::unordered_map<int, unsigned long long> dat_ver_;
  unsigned long long ver_counter_ = 0;
  long long loops_skipped_ = 0;
  bool redundant(const Desc &d, LoopRecord &rec);
  void check_in_allocation(const Desc &d, const Arg &a, const Dat &dt) const;
  long long kernels_launched_ = 0, graphs_launched_ = 0, loops_enqueued_ = 0;
  std::unique_ptr<Transport> transport_;
  std::vector<Slab> slabs_;  // per block, after partition
  bool partitioned_ = false;
  char *stage_h_ = nullptr;  // pinned staging of host-transport exchanges
  size_t stage_cap_ = 0;
  long long exchanges_ = 0;
  long long list_launches_ = 0;  // work lists planned (loops they cover: list_loops_)
  long long list_loops_ = 0;
  std::unordered_map<uint64_t, char *> list_cache_;  // device work lists by content
};

// Releases an app call's declarations (blocks, dats, stencils, reductions
// made after construction) when the scope ends, on the error paths too: a
// driver that throws gives its dat storage back instead of holding it until
// ops_b200_exit. On an error path the queued loops are dropped first, and a
// failure while releasing (a CUDA error that poisoned the context, say) is
// swallowed so that the original error reaches the caller.
class ReleaseScope {
 public:
  explicit ReleaseScope(Runtime &r) : r_(r), m_(r.mark()) {}
  ReleaseScope(const ReleaseScope &) = delete;
  ReleaseScope &operator=(const ReleaseScope &) = delete;
  ~ReleaseScope() {
    if (done_) return;
    try {
      r_.discard_queue();
      r_.release_to(m_);
    } catch (...) {
    }
  }
  // The normal path: release now, errors propagate.
  void release() {
    done_ = true;
    r_.release_to(m_);
  }
  const Runtime::Mark &mark() const { return m_; }

 private:
  Runtime &r_;
  Runtime::Mark m_;
  bool done_ = false;
};

// Two CUDA events (start, end of a timed region) destroyed with the scope.
struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  EventPair() {
    OPSB_CUDA(cudaEventCreate(&a));
    OPSB_CUDA(cudaEventCreate(&b));
  }
  EventPair(const EventPair &) = delete;
  EventPair &operator=(const EventPair &) = delete;
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
  float ms() const {
    float t = 0.f;
    OPSB_CUDA(cudaEventElapsedTime(&t, a, b));
    return t;
  }
};

// ---------------------------------------------------------------------------
// C++ convenience API used by the app drivers (mirrors ops_arg_* and
// ops_par_loop of ops/c/include/ops_lib_core.h / ops_seq_v2.h).
// ---------------------------------------------------------------------------
inline Arg arg_dat(int dat, int dim, int stencil, int acc) {
  Arg a; a.kind = ARG_DAT; a.dat = dat; a.dim = dim; a.stencil = stencil; a.acc = acc; return a;
}
inline Arg arg_dat_opt(int dat, int dim, int stencil, int acc, int flag) {
  Arg a = arg_dat(dat, dim, stencil, acc); a.opt = flag ? 1 : 0; return a;
}
inline Arg arg_gbl(const void *data, int dim, int elem, int acc) {
  Arg a; a.kind = ARG_GBL; a.dim = dim; a.elem = elem; a.acc = acc;
  a.gbl.assign((const char *)data, (const char *)data + (size_t)dim * elem);
  return a;
}
inline Arg arg_reduce(int handle, int dim, int acc) {
  Arg a; a.kind = ARG_REDUCE; a.red = handle; a.dim = dim; a.acc = acc; return a;
}
inline Arg arg_idx() { Arg a; a.kind = ARG_IDX; a.dim = 1; a.elem = 4; return a; }

template <class K>
void launch_exec(const LoopParams &lp, dim3 g, dim3 b, cudaStream_t s) {
  exec_loop<K><<<g, b, 0, s>>>(lp);
}
template <class K>
void launch_exec_list(const LoopParams *items, const ListItem *grids, int n, long long blocks, dim3 b,
                      cudaStream_t s) {
  exec_loop_list<K><<<(unsigned)blocks, b, 0, s>>>(items, grids, n);
}

// A kernel may bring its own launch (a specialised executor for its access
// pattern) as `static void launch(const LoopParams &, dim3, dim3,
// cudaStream_t)`; the runtime's grid shape is passed along as a hint.
template <class K, class = void>
struct CustomLaunch {
  static constexpr bool value = false;
};
template <class K>
struct CustomLaunch<K, std::void_t<decltype(&K::launch)>> {
  static constexpr bool value = true;
};

template <class K, class = void>
struct CopyTrait { static constexpr int dst = -1, src = -1; };
template <class K>
struct CopyTrait<K, std::void_t<decltype(K::copy_dst)>> { static constexpr int dst = K::copy_dst, src = K::copy_src; };

template <class K>
LoopInfo make_loop_info(const char *kernel) {
  LoopInfo li;
  li.kernel = kernel;
  using S = SigInfo<decltype(&K::operator())>;
  li.nparams = S::n;
  S::fill(li.params);
  li.ndim = 0;
  for (int i = 0; i < li.nparams; i++)
    if (li.params[i].cls == 'A') li.ndim = li.params[i].ndim;
  li.copy_dst = CopyTrait<K>::dst;
  li.copy_src = CopyTrait<K>::src;
  if constexpr (CustomLaunch<K>::value) {
    li.launch = &K::launch;
  } else {
    li.launch = &launch_exec<K>;
    li.launch_list = &launch_exec_list<K>;
  }
  li.mgrid_ok = LoopMgridOk<K>::value ? 1 : 0;
  return li;
}

// Registers K under `kernel` at static-initialisation time.
// Registers K under K::kname at static-initialisation time so that the
// C-ABI can launch it by name.
template <class K>
struct LoopRegistrar {
  LoopRegistrar() { Runtime::register_loop(make_loop_info<K>(K::kname)); }
};
#define OPSB_REGISTER_LOOP(K) static ::opsb::LoopRegistrar<K> opsb_reg_##K
template <class K>
struct CopyLoopRegistrar {
  CopyLoopRegistrar() { register_copy_loop(K::kname, K::copy_spec()); }
};
#define OPSB_REGISTER_COPY_LOOP(K) static ::opsb::CopyLoopRegistrar<K> opsb_copy_reg_##K

// ops_par_loop by registered kernel name (what translated app code and the
// C++ app drivers call; no template instantiation at the call site).
inline void par_loop_named(const char *kernel, const char *name, int block, int dim, const int *range,
                           std::initializer_list<Arg> args) {
  const LoopInfo *li = Runtime::find_loop(kernel);
  if (!li) throw Error(E_NOTFOUND, std::string("no registered loop kernel named ") + kernel);
  Runtime::get().par_loop(li, name, block, dim, range, args.begin(), (int)args.size());
}
inline void par_loop_named(const char *kernel, const char *name, int block, int dim, const int *range,
                           const std::vector<Arg> &args) {
  const LoopInfo *li = Runtime::find_loop(kernel);
  if (!li) throw Error(E_NOTFOUND, std::string("no registered loop kernel named ") + kernel);
  Runtime::get().par_loop(li, name, block, dim, range, args.data(), (int)args.size());
}

// Loop kernels of one app looked up once: "<prefix><name>" resolved on the
// first call for a name and kept (keyed by the name's hash, confirmed by
// comparing the text), so the app drivers' per-loop path builds no strings.
class PrefixedLoops {
 public:
  explicit PrefixedLoops(const char *prefix) : prefix_(prefix) {}
  const LoopInfo *get(const char *name) {
    uint64_t h = 0xCBF29CE484222325ULL;
    for (const char *c = name; *c; c++) h = (h ^ (unsigned char)*c) * 0x100000001B3ULL;
    auto it = cache_.find(h);
    if (it != cache_.end() && it->second.first == name) return it->second.second;
    const std::string full = prefix_ + name;
    const LoopInfo *li = Runtime::find_loop(full);
    if (!li) throw Error(E_NOTFOUND, "no registered loop kernel named " + full);
    cache_[h] = {std::string(name), li};
    return li;
  }

 private:
  std::string prefix_;
  std::unordered_map<uint64_t, std::pair<std::string, const LoopInfo *>> cache_;
};

// ops_par_loop(kernel, name, block, dim, range, args...) for a functor K.
template <class K>
void par_loop(const char *name, int block, int dim, const int *range, std::initializer_list<Arg> args) {
  static const LoopInfo *li = nullptr;
  if (!li) {
    li = Runtime::find_loop(K::kname);
    if (!li) {
      static LoopInfo own = make_loop_info<K>(K::kname);
      li = &own;
    }
  }
  Runtime::get().par_loop(li, name, block, dim, range, args.begin(), (int)args.size());
}

}  // namespace opsb
