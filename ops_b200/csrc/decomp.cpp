// Domain decomposition across processes: slab partition of blocks and dats,
// loop clipping, halo exchanges, cross-rank reductions, transports
// (semantics and reference mapping in decomp.h).
#include "decomp.h"

#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>

#include "runtime.h"

namespace opsb {

void slab_bounds(int extent, int nranks, int rank, int *lo, int *hi) {
  // ops_mpi_partition.cpp:236-243: (coord * size) / pdims, with 64-bit
  // products so that large extents times many ranks cannot overflow
  *lo = (int)((long long)rank * extent / nranks);
  *hi = (int)((long long)(rank + 1) * extent / nranks);
}

// ---------------------------------------------------------------------------
// Transports.
// ---------------------------------------------------------------------------
namespace {

class HostTransport : public Transport {
 public:
  HostTransport(int n, int r, const HostCallbacks &cb) : n_(n), r_(r), cb_(cb) {}
  int nranks() const override { return n_; }
  int rank() const override { return r_; }
  bool device() const override { return false; }
  void exchange(const Msg *msgs, int n, cudaStream_t) override {
    if (n == 0) return;
    if (cb_.exchange(cb_.ctx, msgs, n) != 0) throw Error(E_STATE, "halo exchange: the host transport reported an error");
  }
  void allgather(const void *send, size_t bytes, void *recv, cudaStream_t) override {
    if (cb_.allgather(cb_.ctx, send, bytes, recv) != 0)
      throw Error(E_STATE, "reduction: the host transport's allgather reported an error");
  }
  std::string name() const override { return "host"; }

 private:
  int n_, r_;
  HostCallbacks cb_;
};

// NCCL entry points, resolved from libnccl.so.2 (the library already loaded
// into the process, e.g. by PyTorch, when there is one: same soname).
struct NcclApi {
  ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  ncclResult_t (*AllGather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
  const char *(*GetErrorString)(ncclResult_t) = nullptr;
};

const NcclApi &nccl() {
  static NcclApi api;
  static std::once_flag once;
  static std::string err;
  std::call_once(once, [] {
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
      err = std::string("cannot open libnccl.so.2: ") + dlerror();
      return;
    }
    auto sym = [&](const char *n) {
      void *p = dlsym(h, n);
      if (!p && err.empty()) err = std::string("libnccl.so.2 lacks ") + n;
      return p;
    };
    api.GetUniqueId = (decltype(api.GetUniqueId))sym("ncclGetUniqueId");
    api.CommInitRank = (decltype(api.CommInitRank))sym("ncclCommInitRank");
    api.CommDestroy = (decltype(api.CommDestroy))sym("ncclCommDestroy");
    api.Send = (decltype(api.Send))sym("ncclSend");
    api.Recv = (decltype(api.Recv))sym("ncclRecv");
    api.GroupStart = (decltype(api.GroupStart))sym("ncclGroupStart");
    api.GroupEnd = (decltype(api.GroupEnd))sym("ncclGroupEnd");
    api.AllGather = (decltype(api.AllGather))sym("ncclAllGather");
    api.GetErrorString = (decltype(api.GetErrorString))sym("ncclGetErrorString");
  });
  if (!err.empty()) throw Error(E_UNSUPPORTED, "NCCL transport: " + err);
  return api;
}

void nccl_check(ncclResult_t r, const char *what) {
  if (r != ncclSuccess)
    throw Error(E_CUDA, std::string("NCCL error in ") + what + ": " + nccl().GetErrorString(r));
}

class NcclTransport : public Transport {
 public:
  NcclTransport(const void *id, int n, int r) : n_(n), r_(r) {
    ncclUniqueId uid;
    static_assert(sizeof(uid) == 128, "ncclUniqueId is 128 bytes");
    memcpy(&uid, id, sizeof(uid));
    nccl_check(nccl().CommInitRank(&comm_, n, uid, r), "ncclCommInitRank");
  }
  ~NcclTransport() override {
    if (stage_) cudaFree(stage_);
    if (comm_) nccl().CommDestroy(comm_);
  }
  int nranks() const override { return n_; }
  int rank() const override { return r_; }
  bool device() const override { return true; }
  void exchange(const Msg *msgs, int n, cudaStream_t s) override {
    const NcclApi &a = nccl();
    nccl_check(a.GroupStart(), "ncclGroupStart");
    for (int i = 0; i < n; i++) {
      if (msgs[i].peer < 0) continue;
      if (msgs[i].send_bytes)
        nccl_check(a.Send(msgs[i].send, msgs[i].send_bytes, ncclUint8, msgs[i].peer, comm_, s), "ncclSend");
      if (msgs[i].recv_bytes)
        nccl_check(a.Recv(msgs[i].recv, msgs[i].recv_bytes, ncclUint8, msgs[i].peer, comm_, s), "ncclRecv");
    }
    nccl_check(a.GroupEnd(), "ncclGroupEnd");
  }
  void allgather(const void *send, size_t bytes, void *recv, cudaStream_t s) override {
    const size_t need = bytes * (n_ + 1);
    if (need > cap_) {
      if (stage_) OPSB_CUDA(cudaFree(stage_));
      stage_ = nullptr;
      OPSB_CUDA(cudaMalloc(&stage_, need));
      cap_ = need;
    }
    OPSB_CUDA(cudaMemcpyAsync(stage_, send, bytes, cudaMemcpyHostToDevice, s));
    nccl_check(nccl().AllGather(stage_, stage_ + bytes, bytes, ncclUint8, comm_, s), "ncclAllGather");
    OPSB_CUDA(cudaMemcpyAsync(recv, stage_ + bytes, bytes * n_, cudaMemcpyDeviceToHost, s));
    OPSB_CUDA(cudaStreamSynchronize(s));
  }
  std::string name() const override { return "nccl"; }

 private:
  int n_, r_;
  ncclComm_t comm_ = nullptr;
  char *stage_ = nullptr;
  size_t cap_ = 0;
};

}  // namespace

std::unique_ptr<Transport> make_host_transport(int nranks, int rank, const HostCallbacks &cb) {
  if (nranks < 1 || rank < 0 || rank >= nranks) throw Error(E_ARG, "transport: bad rank / number of ranks");
  if (!cb.exchange || !cb.allgather) throw Error(E_ARG, "host transport: both callbacks are required");
  return std::make_unique<HostTransport>(nranks, rank, cb);
}

std::unique_ptr<Transport> make_nccl_transport(const void *unique_id, int nranks, int rank) {
  if (nranks < 1 || rank < 0 || rank >= nranks) throw Error(E_ARG, "transport: bad rank / number of ranks");
  if (!unique_id) throw Error(E_ARG, "NCCL transport: no unique id");
  return std::make_unique<NcclTransport>(unique_id, nranks, rank);
}

void nccl_unique_id(void *out128) {
  ncclUniqueId uid;
  nccl_check(nccl().GetUniqueId(&uid), "ncclGetUniqueId");
  memcpy(out128, &uid, sizeof(uid));
}

// ---------------------------------------------------------------------------
// Runtime: partition.
// ---------------------------------------------------------------------------
#define OPSB_REQUIRE(cond, code, msg)        \
  do {                                       \
    if (!(cond)) throw Error((code), (msg)); \
  } while (0)

void Runtime::set_transport(std::unique_ptr<Transport> t) {
  OPSB_REQUIRE(!partitioned_, E_STATE, "the transport cannot change after ops_partition");
  transport_ = std::move(t);
}

int Runtime::nranks() const { return transport_ ? transport_->nranks() : 1; }
int Runtime::rank() const { return transport_ ? transport_->rank() : 0; }

const Slab &Runtime::slab(int blk) const {
  static const Slab none;
  return (blk >= 0 && blk < (int)slabs_.size()) ? slabs_[blk] : none;
}

// Elements between consecutive indices of dimension k in a dat's storage.
static long long dim_stride(const Dat &d, int k) { return k == 0 ? 1 : (k == 1 ? d.pitch : d.plane); }

// A dat's owned part and window along the split dimension of its block's
// slab (integer arithmetic only; also what the C-ABI's ops_b200_slab_window
// reports).
void slab_window(const Slab &s, int gstart, int gend, int *own_lo, int *own_hi, int *win_lo, int *win_hi) {
  *own_lo = s.first ? gstart : std::max(gstart, s.lo);
  *own_hi = s.last ? gend : std::min(gend, s.hi);
  *win_lo = s.first ? gstart : std::max(gstart, *own_lo - s.halo);
  *win_hi = s.last ? gend : std::min(gend, *own_hi + s.halo);
}

// Moves a dat to its slab window: the rows of the window are copied out of
// the whole-extent storage into a new allocation, whose origin is shifted so
// that global indices address it unchanged.
void Runtime::window_dat(Dat &d) {
  const Slab &s = slabs_[d.block];
  const int k = s.dim;
  if (k < 0 || d.size[k] <= 1) return;  // replicated along the split dimension
  OPSB_REQUIRE(d.locked == 0, E_STATE, "ops_partition: dat " + d.name + " has a raw pointer out");
  const int gstart = d.base[k] + d.d_m[k], gend = gstart + d.size[k];
  int own_lo, own_hi, win_lo, win_hi;
  slab_window(s, gstart, gend, &own_lo, &own_hi, &win_lo, &win_hi);
  OPSB_REQUIRE(own_hi > own_lo, E_UNSUPPORTED,
               "ops_partition: dat " + d.name + " has no points in rank " + std::to_string(rank()) + "'s slab");
  // an inner boundary's halo rows must lie inside the dat (a dat much
  // shorter than its block along the split would end inside a halo)
  OPSB_REQUIRE((s.first || win_lo == own_lo - s.halo) && (s.last || win_hi == own_hi + s.halo), E_UNSUPPORTED,
               "ops_partition: dat " + d.name + " ends within " + std::to_string(s.halo) +
                   " rows of a slab boundary");
  const long long row = dim_stride(d, k);  // elements per index of dimension k
  const size_t row_bytes = (size_t)row * d.elem_size;
  const size_t bytes = row_bytes * (size_t)(win_hi - win_lo);
  char *p = alloc_dat_storage(bytes);
  OPSB_CUDA(cudaMemcpyAsync(p, d.data_d + (size_t)(win_lo - d.lo[k]) * row_bytes, bytes, cudaMemcpyDeviceToDevice,
                            stream_));
  OPSB_CUDA(cudaStreamSynchronize(stream_));
  recycle_dat_storage(d.data_d, d.bytes);
  d.data_d = p;
  d.bytes = bytes;
  d.lo[k] = win_lo;
  d.hi[k] = win_hi;
  d.own_lo[k] = own_lo;
  d.own_hi[k] = own_hi;
  if (k == 1) d.plane = d.pitch * (win_hi - win_lo);
  d.origin = d.pad_front - (long long)d.lo[0] - (long long)d.lo[1] * d.pitch - (long long)d.lo[2] * d.plane;
  d.split = k;
  d.valid = s.halo;  // the window was cut from the whole field: its halo rows are current
  d.host.clear();
}

void Runtime::partition(const char *routine) {
  (void)routine;  // the reference's decomposition-routine name (ops_partition(const char*))
  OPSB_REQUIRE(inited_, E_STATE, "ops_partition before ops_init");
  // blocks declared since the last call (an app call's blocks are released
  // with its other declarations)
  if (nranks() <= 1 || slabs_.size() == blocks_.size()) return;
  execute();
  OPSB_CUDA(cudaStreamSynchronize(stream_));
  // Storage moves: cached graphs, fused plans and shadows refer to the old one.
  for (auto &kv : graphs_)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  graphs_.clear();
  release_fusion_plans();
  for (auto &kv : shadow_)
    if (kv.second) recycle_dat_storage(kv.second, dats_[kv.first]->bytes);
  shadow_.clear();
  const int N = nranks(), R = rank();
  const size_t first_new = slabs_.size();
  slabs_.resize(blocks_.size());
  for (size_t bi = first_new; bi < blocks_.size(); bi++) {
    const Block &b = blocks_[bi];
    Slab &s = slabs_[b.index];
    if (b.dims < 2) continue;  // 1D blocks are replicated
    const int k = b.dims - 1;
    int extent = 0;
    for (auto &dp : dats_)
      if (dp && dp->block == b.index)
        extent = std::max(extent, dp->size[k] + dp->base[k] + dp->d_m[k] - dp->d_p[k]);
    int halo = 0;
    for (const Stencil &st : stencils_) {
      if (st.dims != b.dims || st.stride[k] == 0 || st.type != 0) continue;
      for (int p = 0; p < st.points; p++) halo = std::max(halo, std::abs(st.offs[(size_t)p * st.dims + k]));
    }
    OPSB_REQUIRE(extent / N >= std::max(halo, 1), E_UNSUPPORTED,
                 "ops_partition: block " + b.name + " is " + std::to_string(extent) + " along dimension " +
                     std::to_string(k) + ", too thin for " + std::to_string(N) + " slabs of at least " +
                     std::to_string(std::max(halo, 1)) + " rows");
    s.dim = k;
    s.extent = extent;
    s.halo = halo;
    s.first = R == 0;
    s.last = R == N - 1;
    slab_bounds(extent, N, R, &s.lo, &s.hi);
  }
  for (auto &dp : dats_)
    if (dp && dp->block >= (int)first_new) window_dat(*dp);
  partitioned_ = true;
}

// ---------------------------------------------------------------------------
// Runtime: loops on a partitioned block.
// ---------------------------------------------------------------------------
// Clips a loop's range to this rank's slab when it touches a partitioned dat
// (compute_ranges in the reference's MPI backend); loops over replicated
// dats only run in full on every rank.
void Runtime::clip_loop(Desc &d) {
  if (!partitioned_) return;
  const Slab &s = slab(d.block);
  if (s.dim < 0) return;
  const int k = s.dim;
  bool touches = false;
  for (const Arg &a : d.args) {
    if (a.kind != ARG_DAT) continue;
    const Dat &dt = dat(a.dat);
    const Stencil &st = stencil(a.stencil);
    if (dt.split < 0) continue;
    OPSB_REQUIRE(st.type == 0, E_UNSUPPORTED,
                 "loop " + d.loop->kernel + ": restrict/prolong stencils on a partitioned block");
    OPSB_REQUIRE(st.stride[k] != 0, E_UNSUPPORTED,
                 "loop " + d.loop->kernel + ": dat " + dt.name +
                     " is partitioned but read through a stencil folded along the split dimension");
    touches = true;
  }
  if (!touches) {
    // every rank runs it whole: a sum into a reduction would count it once per rank
    for (const Arg &a : d.args)
      OPSB_REQUIRE(!(a.kind == ARG_REDUCE && a.acc == ACC_INC), E_UNSUPPORTED,
                   "loop " + d.loop->kernel + " sums into a reduction but touches no partitioned dat");
    return;
  }
  int lo = d.range[2 * k], hi = d.range[2 * k + 1];
  if (!s.first) lo = std::max(lo, s.lo);
  if (!s.last) hi = std::min(hi, s.hi);
  d.range[2 * k] = lo;
  d.range[2 * k + 1] = std::max(lo, hi);
}

// Before a loop that reads a partitioned dat across the slab boundary
// through its stencil, the neighbours' rows are brought in if the dat was
// written since its last exchange (ops_halo_exchanges with dirty bits,
// ops_mpi_rt_support.cpp:836). The decision uses only the stencils and the
// write history, so every rank makes it identically. Afterwards the dats the
// loop writes are marked as changed.
void Runtime::exchange_for_loop(const Desc &d) {
  if (!partitioned_) return;
  const Slab &s = slab(d.block);
  if (s.dim < 0) return;
  const int k = s.dim;
  std::vector<int> need;
  for (const Arg &a : d.args) {
    if (a.kind != ARG_DAT || a.acc == ACC_WRITE) continue;
    Dat &dt = dat(a.dat);
    if (dt.split < 0) continue;
    const Stencil &st = stencil(a.stencil);
    int reach = 0;
    for (int p = 0; p < st.points; p++) reach = std::max(reach, std::abs(st.offs[(size_t)p * st.dims + k]));
    if (reach > 0 && dt.valid < reach && std::find(need.begin(), need.end(), a.dat) == need.end())
      need.push_back(a.dat);
  }
  if (!need.empty()) exchange_dats(need);
}

void Runtime::mark_written(const Desc &d) {
  if (!partitioned_) return;
  for (const Arg &a : d.args)
    if (a.kind == ARG_DAT && a.acc != ACC_READ) {
      Dat &dt = *dats_[a.dat];
      if (dt.split >= 0) dt.valid = 0;
    }
}

namespace {
// The runtime-internal queue item of an exchange (NCCL transport).
LoopInfo &exchange_info() {
  static LoopInfo li = [] {
    LoopInfo l;
    l.kernel = "__halo_exchange";
    l.internal = 2;
    return l;
  }();
  return li;
}
}  // namespace

// The messages of one exchange of `dats` (whole halo depth of their slab):
// per neighbour, per dat, the owned rows next to it out and the rows beyond
// the boundary in. `base(d)` gives where a dat's storage starts in the
// memory space the messages use.
template <class Base>
static std::vector<Msg> exchange_msgs(const std::vector<Dat *> &dats, const Slab &s, int rank, Base base) {
  std::vector<Msg> m;
  for (int side = 0; side < 2; side++) {
    const bool has = side == 0 ? !s.first : !s.last;
    if (!has) continue;
    const int peer = side == 0 ? rank - 1 : rank + 1;
    for (Dat *d : dats) {
      const int k = d->split;
      const size_t row = (size_t)dim_stride(*d, k) * d->elem_size;
      const int h = s.halo;
      // lower side: send [own_lo, own_lo+h), receive [own_lo-h, own_lo);
      // upper side: send [own_hi-h, own_hi), receive [own_hi, own_hi+h)
      const int send0 = side == 0 ? d->own_lo[k] : d->own_hi[k] - h;
      const int recv0 = side == 0 ? d->own_lo[k] - h : d->own_hi[k];
      Msg x;
      x.peer = peer;
      x.send = base(*d) + (size_t)(send0 - d->lo[k]) * row;
      x.send_bytes = row * h;
      x.recv = base(*d) + (size_t)(recv0 - d->lo[k]) * row;
      x.recv_bytes = row * h;
      m.push_back(x);
    }
  }
  return m;
}

void Runtime::exchange_dats(const std::vector<int> &ids) {
  const Slab &s = slab(dat(ids[0]).block);
  std::vector<Dat *> dats;
  for (int i : ids) {
    Dat &d = dat(i);
    // both neighbours' windows hold the same rows: the receiving halo and
    // the sent owned rows have equal row sizes on both sides
    OPSB_REQUIRE(d.own_hi[d.split] - d.own_lo[d.split] >= s.halo, E_UNSUPPORTED,
                 "halo exchange: dat " + d.name + " owns fewer rows than the halo depth");
    dats.push_back(&d);
  }
  exchanges_++;
  if (transport_->device()) {
    // queued with the loops: NCCL send/recv on the runtime stream, captured
    // into the flush's graph like a kernel
    Desc x;
    x.loop = &exchange_info();
    x.name = "__halo_exchange";
    x.block = dats[0]->block;
    x.dim = blocks_[x.block].dims;
    for (Dat *d : dats) {
      Arg a;
      a.kind = ARG_DAT;
      a.dat = d->index;
      a.stencil = 0;
      a.acc = ACC_RW;
      x.args.push_back(a);
    }
    x.red_first.assign(x.args.size(), 0);
    x.gbl_off.assign(x.args.size(), 0);
    queue_.push_back(std::move(x));
    qrec_.push_back(LoopRecord());
    for (Dat *d : dats) d->valid = s.halo;
    return;
  }
  // host transport: run the queue, stage the sent rows through pinned
  // memory (one message per neighbour: every dat's rows back to back), let
  // the caller move them, put the received rows in place
  execute();
  std::vector<Msg> dev = exchange_msgs(dats, s, rank(), [](const Dat &d) { return d.data_d; });
  size_t total = 0;
  for (const Msg &m : dev) total += m.send_bytes + m.recv_bytes;
  if (total > stage_cap_) {
    if (stage_h_) OPSB_CUDA(cudaFreeHost(stage_h_));
    stage_h_ = nullptr;
    OPSB_CUDA(cudaMallocHost(&stage_h_, total));
    stage_cap_ = total;
  }
  std::vector<Msg> host;        // per neighbour
  std::vector<char *> recv_at;  // per device message: its rows in the staging buffer
  size_t off = 0;
  for (size_t i = 0; i < dev.size();) {
    size_t j = i;
    size_t sb = 0, rb = 0;
    while (j < dev.size() && dev[j].peer == dev[i].peer) {
      sb += dev[j].send_bytes;
      rb += dev[j].recv_bytes;
      j++;
    }
    Msg h;
    h.peer = dev[i].peer;
    h.send = stage_h_ + off;
    h.send_bytes = sb;
    h.recv = stage_h_ + off + sb;
    h.recv_bytes = rb;
    size_t so = off, ro = off + sb;
    for (size_t q = i; q < j; q++) {
      OPSB_CUDA(cudaMemcpyAsync(stage_h_ + so, dev[q].send, dev[q].send_bytes, cudaMemcpyDeviceToHost, stream_));
      so += dev[q].send_bytes;
      recv_at.push_back(stage_h_ + ro);
      ro += dev[q].recv_bytes;
    }
    off += sb + rb;
    host.push_back(h);
    i = j;
  }
  OPSB_CUDA(cudaStreamSynchronize(stream_));
  transport_->exchange(host.data(), (int)host.size(), stream_);
  for (size_t i = 0; i < dev.size(); i++)
    OPSB_CUDA(cudaMemcpyAsync(dev[i].recv, recv_at[i], dev[i].recv_bytes, cudaMemcpyHostToDevice, stream_));
  OPSB_CUDA(cudaStreamSynchronize(stream_));
  for (Dat *d : dats) {
    d->valid = s.halo;
    d->host.clear();
  }
}

// The queued exchange item (NCCL transport), resolved at planning time.
PlanItem Runtime::prepare_exchange(const Desc &x) {
  std::vector<Dat *> dats;
  for (const Arg &a : x.args) dats.push_back(dats_[a.dat].get());
  const Slab &s = slab(x.block);
  std::vector<Msg> msgs = exchange_msgs(dats, s, rank(), [](const Dat &d) { return d.data_d; });
  PlanItem it;
  it.name = "runtime/halo_exchange";
  for (const Msg &m : msgs) it.bytes += (double)(m.send_bytes + m.recv_bytes);
  Transport *t = transport_.get();
  it.run = [t, msgs](cudaStream_t st) { t->exchange(msgs.data(), (int)msgs.size(), st); };
  return it;
}

// ---------------------------------------------------------------------------
// Runtime: reductions across ranks.
// ---------------------------------------------------------------------------
namespace {
template <class T>
void combine(T *acc, const T *v, int n, int op) {
  for (int i = 0; i < n; i++) {
    if (op == ACC_INC)
      acc[i] = acc[i] + v[i];
    else if (op == ACC_MIN)
      acc[i] = v[i] < acc[i] ? v[i] : acc[i];
    else if (op == ACC_MAX)
      acc[i] = v[i] > acc[i] ? v[i] : acc[i];
  }
}
}  // namespace

// Every rank's value of the handle, combined in rank order: (r0 op r1) op r2
// ..., the same bits on every rank and from run to run.
void Runtime::combine_reduction(const Reduction &r, void *value) {
  const int N = nranks();
  std::vector<char> all((size_t)r.size * N);
  transport_->allgather(value, (size_t)r.size, all.data(), stream_);
  std::vector<char> acc(all.begin(), all.begin() + r.size);
  for (int q = 1; q < N; q++) {
    const char *v = all.data() + (size_t)q * r.size;
    const int n = r.size / std::max(1, r.elem);
    const std::string &t = r.type;
    if (t == "double")
      combine((double *)acc.data(), (const double *)v, n, r.acc);
    else if (t == "float")
      combine((float *)acc.data(), (const float *)v, n, r.acc);
    else if (t == "int")
      combine((int *)acc.data(), (const int *)v, n, r.acc);
    else if (t == "unsigned int")
      combine((unsigned int *)acc.data(), (const unsigned int *)v, n, r.acc);
    else if (t == "long" || t == "long long" || t == "ll")
      combine((long long *)acc.data(), (const long long *)v, n, r.acc);
    else if (t == "short")
      combine((short *)acc.data(), (const short *)v, n, r.acc);
    else if (t == "char")
      combine((signed char *)acc.data(), (const signed char *)v, n, r.acc);
    else
      throw Error(E_UNSUPPORTED, "reduction " + r.name + ": type " + t + " cannot be combined across ranks");
  }
  memcpy(value, acc.data(), r.size);
}

}  // namespace opsb
