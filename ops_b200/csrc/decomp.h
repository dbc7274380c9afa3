// Domain decomposition across processes (ops_partition): one process per
// GPU, each owning a slab of every block along the block's outermost
// dimension (y in 2D, z in 3D).
//
// Reference behaviour (ops/c/src/mpi/): ops_partition_blocks splits a block's
// extent, the largest interior size + base of its dats
// (ops_mpi_partition.cpp:84-256), into equal pieces by integer division;
// ops_decomp (:257) gives each process its piece and its neighbours; every
// loop runs over the intersection of its range with the owned piece
// (ops_mpi_rt_support.cpp compute_ranges); ops_halo_exchanges (:836) brings
// in the neighbours' rows a loop's stencils read when they changed since the
// last exchange (dirty bits); reductions are combined across processes
// (ops_mpi_reduce_*, :1271-1307).
//
// B200 design:
//   * Slabs along the outermost dimension only, so every halo is a run of
//     whole pitched rows (2D) or planes (3D): contiguous memory, one send
//     and one receive per neighbour straight between the dats' storage, no
//     pack or unpack kernels. Loop indices stay global: a partitioned dat is
//     a smaller allocation whose origin is shifted, so stencil offsets,
//     accessors and every executor are unchanged.
//   * Dats of extent 1 along the split dimension (edge dats such as
//     CloverLeaf's cellx) are replicated, and loops that touch no
//     partitioned dat run in full on every process.
//   * Exchanges are decided from global information only (the loop's
//     stencils and the dats' write history, identical on every process), so
//     all processes take the same exchange steps in the same order.
//   * Reduction results are gathered and combined in rank order on the
//     host: sums are reproducible from run to run and equal on every rank.
//   * Transport: a host transport (the caller moves host buffers, e.g. over
//     gloo; the runtime stages rows through pinned memory and flushes its
//     queue first) or NCCL (ncclSend/ncclRecv on the runtime's stream, queued
//     with the loops).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <memory>
#include <string>
#include <vector>

namespace opsb {

// One point-to-point transfer of an exchange: `send_bytes` from `send` to
// rank `peer` and `recv_bytes` from `peer` into `recv` (either may be 0).
struct Msg {
  int peer = -1;
  const void *send = nullptr;
  size_t send_bytes = 0;
  void *recv = nullptr;
  size_t recv_bytes = 0;
};

class Transport {
 public:
  virtual ~Transport() = default;
  virtual int nranks() const = 0;
  virtual int rank() const = 0;
  // Buffers of `exchange` are device memory and the transfers are ordered on
  // `stream` (true), or host memory and complete on return (false).
  virtual bool device() const = 0;
  virtual void exchange(const Msg *msgs, int n, cudaStream_t stream) = 0;
  // Every rank's `bytes` from `send`, in rank order, into `recv` (host
  // memory; complete on return).
  virtual void allgather(const void *send, size_t bytes, void *recv, cudaStream_t stream) = 0;
  virtual std::string name() const = 0;
};

// Host transport over two caller functions (the C-ABI's
// ops_b200_exchange_fn / ops_b200_allgather_fn): each returns 0 on success.
struct HostCallbacks {
  int (*exchange)(void *ctx, const Msg *msgs, int n) = nullptr;
  int (*allgather)(void *ctx, const void *send, size_t bytes, void *recv) = nullptr;
  void *ctx = nullptr;
};
std::unique_ptr<Transport> make_host_transport(int nranks, int rank, const HostCallbacks &cb);

// NCCL transport (libnccl.so.2 opened at run time). `unique_id` is the
// 128-byte ncclUniqueId that rank 0 made with nccl_unique_id and every rank
// received; the communicator is bound to the runtime's current device.
std::unique_ptr<Transport> make_nccl_transport(const void *unique_id, int nranks, int rank);
void nccl_unique_id(void *out128);

// The slab of one block a rank owns along the split dimension, in the
// block's logical index space (`lo` of rank 0 and `hi` of the last rank are
// open: they also own the halos beyond the interior).
struct Slab {
  int dim = -1;            // split dimension (-1: the block is not split)
  int extent = 0;          // block extent along it: max over dats of interior size + base
  int lo = 0, hi = 0;      // owned [lo, hi) of the interior
  int first = 1, last = 1; // this rank holds the lower / upper end
  int halo = 0;            // rows (planes) of neighbour data each partitioned dat keeps
};

// ops_partition_blocks' equal division (integer division of the extent by
// the ranks): rank r owns [r*extent/nranks, (r+1)*extent/nranks).
void slab_bounds(int extent, int nranks, int rank, int *lo, int *hi);

// A dat spanning [gstart, gend) along the split dimension: the part this
// rank owns (computes, fetches and sends) and the window it stores (the
// owned part and `halo` rows of each neighbour's).
void slab_window(const Slab &s, int gstart, int gend, int *own_lo, int *own_hi, int *win_lo, int *win_hi);

}  // namespace opsb
