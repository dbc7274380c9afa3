"""Decomposition across processes (one process per GPU) over torch.distributed.

The reference runs a partitioned OPS application as MPI ranks
(ops/c/src/mpi/): ops_partition splits every block, loops run over their
rank's part, halos are exchanged and reductions combined. OPS-B200 splits
each 2D/3D block into slabs along its outermost dimension
(include/ops_b200.h, "Decomposition across processes"); this module gives the
runtime its transport:

* ``use_host_transport(group)``: the runtime stages the halo rows through
  pinned host memory and this module moves them with torch.distributed
  point-to-point calls (gloo, or any backend that sends CPU tensors), and
  gathers reduction values with all_gather. Works with several processes on
  one GPU (the exchange is host-synchronous: no kernel waits on another
  process).
* ``use_nccl_transport(group)``: NCCL inside the library; rank 0's 128-byte
  unique id is broadcast through the group, and exchanges become
  ncclSend/ncclRecv on the runtime stream, queued and graph-captured with
  the loops. NCCL needs one GPU per rank.

Set the transport before the app's declarations reach ops_partition (the app
drivers call it where the reference apps do). Every rank then issues the same
calls in the same order.
"""
import ctypes

import torch
import torch.distributed as dist

from ._lib import ALLGATHER_FN, EXCHANGE_FN, check, lib

_active = []  # the transport whose callbacks the library holds


def _host_view(ptr, nbytes):
    """A uint8 CPU tensor over `nbytes` of host memory at `ptr` (no copy)."""
    if nbytes == 0:
        return torch.empty(0, dtype=torch.uint8)
    return torch.frombuffer((ctypes.c_uint8 * nbytes).from_address(ptr), dtype=torch.uint8)


class HostTransport:
    """Halo rows and reduction values moved through host memory by a
    torch.distributed process group."""

    def __init__(self, group=None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.error = None
        self._ex = EXCHANGE_FN(self._exchange)
        self._ag = ALLGATHER_FN(self._allgather)

    def _global(self, r):
        return r if self.group is None else dist.get_global_rank(self.group, r)

    def _exchange(self, ctx, msgs, n):
        try:
            works = []
            recvs = []
            for i in range(n):
                m = msgs[i]
                if m.send_bytes:
                    works.append(dist.isend(_host_view(m.send, m.send_bytes), self._global(m.peer), group=self.group))
                if m.recv_bytes:
                    recvs.append(dist.irecv(_host_view(m.recv, m.recv_bytes), self._global(m.peer), group=self.group))
            for w in recvs + works:
                w.wait()
            return 0
        except Exception as e:  # reported to the runtime, which raises
            self.error = e
            return -1

    def _allgather(self, ctx, send, nbytes, recv):
        try:
            src = _host_view(send, nbytes).clone()
            parts = [torch.empty(nbytes, dtype=torch.uint8) for _ in range(self.size)]
            dist.all_gather(parts, src, group=self.group)
            dst = _host_view(recv, nbytes * self.size)
            for q, p in enumerate(parts):
                dst[q * nbytes:(q + 1) * nbytes] = p
            return 0
        except Exception as e:
            self.error = e
            return -1


def use_host_transport(group=None):
    """Partition across the ranks of `group` with the host transport."""
    t = HostTransport(group)
    check(lib().ops_b200_set_transport_host(t.size, t.rank, t._ex, t._ag, None))
    _active[:] = [t]
    return t


def use_nccl_transport(group=None):
    """Partition across the ranks of `group` with NCCL (one GPU per rank);
    call after ops_init on the rank's device."""
    rank, size = dist.get_rank(group), dist.get_world_size(group)
    uid = (ctypes.c_uint8 * 128)()
    if rank == 0:
        check(lib().ops_b200_nccl_unique_id(ctypes.addressof(uid)))
    obj = [bytes(uid)]
    src = 0 if group is None else dist.get_global_rank(group, 0)
    dist.broadcast_object_list(obj, src=src, group=group)
    ctypes.memmove(ctypes.addressof(uid), obj[0], 128)
    check(lib().ops_b200_set_transport_nccl(ctypes.addressof(uid), size, rank))
    _active[:] = []


def rank_info():
    """(rank, nranks, halo exchanges made so far) of this process's runtime."""
    r, n, e = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
    check(lib().ops_b200_rank_info(ctypes.byref(r), ctypes.byref(n), ctypes.byref(e)))
    return r.value, n.value, e.value


def slab_window(extent, nranks, rank, halo, gstart, gend):
    """The slab arithmetic of ops_partition for one rank (no GPU): the owned
    interior [lo, hi) of a block of `extent` and, for a dat spanning [gstart,
    gend) along the split, its owned part and stored window."""
    v = [ctypes.c_int() for _ in range(6)]
    check(lib().ops_b200_slab_window(extent, nranks, rank, halo, gstart, gend, *[ctypes.byref(x) for x in v]))
    lo, hi, own_lo, own_hi, win_lo, win_hi = (x.value for x in v)
    return {"lo": lo, "hi": hi, "own": (own_lo, own_hi), "window": (win_lo, win_hi)}


def transport_selftest():
    """Exchange a pattern with the neighbours and gather the ranks through
    the library's transport path (no GPU); raises on a mismatch."""
    check(lib().ops_b200_transport_selftest())


def assign_by_cost(costs, nparts):
    """Independent work units (the blocks of a batched tridiagonal solve) over
    `nparts` ranks by cost, longest first onto the least loaded rank (ties:
    the lower rank, then the lower unit index), so every rank computes the
    same assignment without communicating. Returns one ascending list of unit
    indices per rank; the heaviest load is at most 4/3 of the optimum plus
    one unit (Graham's bound for this rule)."""
    if nparts < 1:
        raise ValueError("nparts must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * nparts
    parts = [[] for _ in range(nparts)]
    for i in order:
        r = min(range(nparts), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]
