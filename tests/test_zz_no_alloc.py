"""The allocation-free Laplace sweep (ops_b200_laplace_sweep_noalloc).

It exists for callers that cannot allocate device memory where they need a
sweep (a memory pool owned by another framework, a stream capture that must
not gain allocation nodes, latency-critical loops). The test calls it through
the C-ABI twice in a row on caller-owned buffers and checks each result bit
for bit against the allocating entry point (ops_b200_app_laplace2d) run for
one and for two iterations: the fixed scratch array must give the same
answer on every call, including the second one that reuses it.

Named test_zz_* so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

from ops_b200 import apps, lib, seeded

pytestmark = pytest.mark.gpu


def _bind():
    L = lib()
    f = L.ops_b200_laplace_sweep_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    L.ops_b200_noalloc_last_error.restype = ctypes.c_char_p
    return f, L


# (300, 5000): the grid's y extent is clamped (790 blocks of 2 rows), so the
# kernel's y loop makes several passes; (65536, 40): the widest allowed
# rows, 512 blocks across, where the block budget of the shared scratch
# bounds the grid's y extent.
@pytest.mark.parametrize("imax,jmax,seed", [(300, 211, 3), (4096, 64, 4), (1, 1, 5), (300, 5000, 6),
                                            (65536, 40, 7)])
def test_noalloc_sweep_matches_allocating_entry_point(imax, jmax, seed):
    import torch
    sweep, L = _bind()
    init = seeded.laplace_field(imax, jmax, seed)
    W = imax + 2
    dev = torch.device("cuda:0")
    torch.cuda.set_device(0)
    bufs = [torch.from_numpy(init.copy()).to(dev), torch.from_numpy(init.copy()).to(dev)]
    err = torch.zeros(2, dtype=torch.float64, device=dev)
    origin = lambda t: t.data_ptr() + (W + 1) * 8  # logical (0, 0)
    stream = torch.cuda.current_stream().cuda_stream
    # call 1: buf0 -> buf1; call 2: buf1 -> buf0 (two calls in a row share the scratch)
    assert sweep(imax, jmax, origin(bufs[0]), origin(bufs[1]), W, err.data_ptr(), stream) == 0, \
        L.ops_b200_noalloc_last_error()
    assert sweep(imax, jmax, origin(bufs[1]), origin(bufs[0]), W, err.data_ptr() + 8, stream) == 0, \
        L.ops_b200_noalloc_last_error()
    torch.cuda.synchronize()
    got1 = bufs[1].cpu().numpy()
    got2 = bufs[0].cpu().numpy()
    e = err.cpu().numpy()
    ref1, errs1, _ = apps.laplace2d(init, 1)
    ref2, errs2, _ = apps.laplace2d(init, 2)
    assert np.array_equal(got1, ref1)
    assert np.array_equal(got2, ref2)
    assert e[0] == errs1[0] and e[1] == errs2[1]


def test_noalloc_rejects_oversize():
    sweep, L = _bind()
    import torch
    x = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    rc = sweep(65537, 4, x.data_ptr(), x.data_ptr(), 65539, x.data_ptr(), None)
    assert rc == -1
    assert b"65536" in L.ops_b200_noalloc_last_error()
