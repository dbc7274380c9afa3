"""Decomposition across processes, host side (no GPU).

* The slab arithmetic of ops_partition (ops_b200_slab_window): the reference's
  integer division of a block's extent (ops/c/src/mpi/ops_mpi_partition.cpp:
  236-243), each dat's owned part and stored window.
* The library's host transport path driven by gloo ranks (world size 2 and 3,
  so that an inner rank has two neighbours): halo messages from the C++
  runtime through ops_b200.dist's callbacks to torch.distributed and back,
  and the rank-ordered all-gather that reductions combine from.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("extent,nranks", [(70, 2), (70, 3), (133, 8), (7, 7), (1000, 6)])
def test_slabs_tile_the_extent(opsb_lib, extent, nranks):
    from ops_b200 import dist as D
    prev = 0
    for r in range(nranks):
        w = D.slab_window(extent, nranks, r, 2, -2, extent + 2)
        assert w["lo"] == prev and w["hi"] == (r + 1) * extent // nranks
        prev = w["hi"]
    assert prev == extent


@pytest.mark.parametrize("nranks,halo", [(2, 2), (3, 4), (5, 1)])
def test_dat_windows(opsb_lib, nranks, halo):
    """A dat of CloverLeaf's shape along y: 64 cells, d_m = -2, d_p = 2 (vol_flux_y
    has one more row): the owned parts tile the dat, the first and last ranks
    own the physical halos, and each window is the owned part widened by the
    halo depth towards every neighbour."""
    from ops_b200 import dist as D
    extent = 64 + 6
    for gstart, gend in ((-2, 69 + 2), (-2, 70 + 2)):
        owned = []
        for r in range(nranks):
            w = D.slab_window(extent, nranks, r, halo, gstart, gend)
            lo, hi = w["own"]
            wl, wh = w["window"]
            owned.append((lo, hi))
            assert wl == (gstart if r == 0 else lo - halo)
            assert wh == (gend if r == nranks - 1 else hi + halo)
        assert owned[0][0] == gstart and owned[-1][1] == gend
        for a, b in zip(owned, owned[1:]):
            assert a[1] == b[0]


RANK_SCRIPT = r"""
import json, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{port}", rank={rank}, world_size={world})
from ops_b200 import dist as D
D.use_host_transport()
D.transport_selftest()
r, n, e = D.rank_info()
dist.barrier()
dist.destroy_process_group()
print("RESULT " + json.dumps({{"rank": r, "nranks": n}}))
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(240)
@pytest.mark.parametrize("world", [2, 3])
def test_host_transport_gloo(opsb_lib, world):
    port = free_port()
    procs = []
    for r in range(world):
        code = RANK_SCRIPT.format(root=ROOT, port=port, rank=r, world=world)
        env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    seen = set()
    for p in procs:
        o, e = p.communicate(timeout=200)
        assert p.returncode == 0, e[-3000:]
        res = json.loads([l for l in o.splitlines() if l.startswith("RESULT ")][-1][len("RESULT "):])
        assert res["nranks"] == world
        seen.add(res["rank"])
    assert seen == set(range(world))


@pytest.mark.parametrize("nranks", [1, 2, 3, 4, 8])
def test_tridiagonal_batch_blocks_by_cost(nranks):
    """The 64 uneven blocks of the batched tridiagonal workload (edges
    log-uniform in [32, 192]) go to ranks by cost, longest first onto the
    least loaded: every block exactly once, the same answer on every call,
    and the heaviest rank within Graham's LPT bound of the optimum."""
    import numpy as np

    import bench
    from ops_b200.dist import assign_by_cost
    costs = [int(np.prod(s)) for s in bench.adi_batch_shapes()]
    parts = assign_by_cost(costs, nranks)
    assert len(parts) == nranks
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    assert parts == assign_by_cost(costs, nranks)
    loads = [sum(costs[i] for i in p) for p in parts]
    opt = max(sum(costs) / nranks, max(costs))
    assert max(loads) <= (4.0 / 3.0 - 1.0 / (3 * nranks)) * opt + 1e-9 * opt
