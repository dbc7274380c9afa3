"""Batched tridiagonal solves on the B200 path vs the CPU oracle (Thomas).

Two kernels: strided sweeps (y, z) run Thomas per line; x sweeps split
each line into chunks (partition method), whose rounding differs from
sequential Thomas. FP64 results agree to 1e-12 relative, FP32 to 2e-4; the
FP64 residual of the solved system is checked at full size."""
import ctypes

import numpy as np
import pytest

from ops_b200 import ops as O
from ops_b200 import seeded

pytestmark = pytest.mark.gpu


def oracle_solve(orc, a, b, c, d, solvedim, u=None):
    nd = a.ndim
    dims = (ctypes.c_int * 3)(*list(reversed(a.shape)), *([1] * (3 - nd)))
    f = orc.oracle_trid_batch_d if a.dtype == np.float64 else orc.oracle_trid_batch_s
    f(a.ctypes.data, b.ctypes.data, c.ctypes.data, d.ctypes.data, None if u is None else u.ctypes.data, nd,
      solvedim, dims, dims)


def padded(t, pad):
    """Copy t into a larger zero array (numpy order) and return the device
    tensor plus the offset view description."""
    import torch
    big = np.zeros(tuple(s + p for s, p in zip(t.shape, pad)), dtype=t.dtype)
    big[tuple(slice(0, s) for s in t.shape)] = t
    return torch.from_numpy(big).cuda()


def run_gpu(a, b, c, d, solvedim, u=None, pad=None):
    import torch
    pad = pad or (0,) * a.ndim
    tens = [padded(t, pad) for t in (a, b, c, d)]
    ut = padded(u, pad) if u is not None else None
    shape_p = tens[0].shape
    dims = list(reversed(a.shape))
    pads = list(reversed(shape_p))
    sysd = dict(a=tens[0].data_ptr(), b=tens[1].data_ptr(), c=tens[2].data_ptr(), d=tens[3].data_ptr(),
                u=ut.data_ptr() if ut is not None else None, dims=dims, pads=pads)
    O.trid_batch(a.itemsize, solvedim, [sysd], None)
    torch.cuda.synchronize()
    sl = tuple(slice(0, s) for s in a.shape)
    return tens[3].cpu().numpy()[sl], (ut.cpu().numpy()[sl] if ut is not None else None)


@pytest.mark.parametrize("dtype,rtol", [(np.float64, 1e-12), (np.float32, 2e-4)])
@pytest.mark.parametrize("solvedim", [0, 1, 2])
@pytest.mark.parametrize("shape,pad", [((23, 29, 37), (0, 2, 3)), ((3, 300, 17), (1, 0, 5)), ((9, 8, 256), (0, 0, 0))])
def test_strided_batch_matches_oracle(gpu_runtime, orc, dtype, rtol, solvedim, shape, pad):
    if solvedim == 0 and shape[2] > 512:
        pytest.skip("x line longer than the tile kernel's maximum")
    a, b, c, d = seeded.trid_system(shape, solvedim, 11, dtype)
    x, _ = run_gpu(a, b, c, d, solvedim, pad=pad)
    ref = d.copy()
    oracle_solve(orc, a, b, c, ref, solvedim)
    np.testing.assert_allclose(x, ref, rtol=rtol, atol=rtol * np.abs(ref).max())


@pytest.mark.parametrize("dtype,rtol", [(np.float64, 1e-12), (np.float32, 2e-4)])
@pytest.mark.parametrize("n,inc", [(1, False), (8, False), (37, True), (130, False), (16, True)])
def test_many_x_lines_match_oracle(gpu_runtime, orc, dtype, rtol, n, inc):
    """x sweeps over 20012 lines of one to 130 rows (many tiles of the
    partition kernel), padding and the _Inc form against the oracle."""
    shape = (4, 5003, n)
    a, b, c, d = seeded.trid_system(shape, 0, 21 + n, dtype)
    u = seeded.uniform(5, np.arange(d.size, dtype=np.uint64), -1, 1).reshape(d.shape).astype(dtype) if inc else None
    dg, ug = run_gpu(a, b, c, d, 0, u=u, pad=(0, 1, 3))
    ref = d.copy()
    oracle_solve(orc, a, b, c, ref, 0)
    if inc:
        assert np.array_equal(dg, d)
        np.testing.assert_allclose(ug, u + ref, rtol=rtol, atol=rtol * np.abs(ref).max())
    else:
        np.testing.assert_allclose(dg, ref, rtol=rtol, atol=rtol * np.abs(ref).max())


@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_inc_form(gpu_runtime, orc, solvedim):
    a, b, c, d = seeded.trid_system((11, 13, 70), solvedim, 4)
    u = seeded.uniform(9, np.arange(d.size, dtype=np.uint64), -1, 1).reshape(d.shape)
    dg, ug = run_gpu(a, b, c, d, solvedim, u=u)
    assert np.array_equal(dg, d)
    ref = d.copy()
    oracle_solve(orc, a, b, c, ref, solvedim)
    np.testing.assert_allclose(ug, u + ref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 15, 16, 17, 31, 63, 64, 65, 127, 128, 129, 200, 255, 256, 257, 700])
@pytest.mark.parametrize("solvedim", [0, 1])
@pytest.mark.parametrize("warp", [-1, 0, 1])
def test_line_lengths(gpu_runtime, orc, n, solvedim, warp):
    """x lines: the warp-per-line kernel (4 or 8 rows a lane, lines up to
    256 rows) and the shared-memory tile kernel, each forced and as chosen
    by line length; y lines: the line kernel."""
    if solvedim == 1 and warp != -1:
        pytest.skip("the option steers x sweeps only")
    shape = (5, n) if solvedim == 0 else (n, 7)
    a, b, c, d = seeded.trid_system(shape, solvedim, n)
    O.set_option("trid_warp", warp)
    try:
        x, _ = run_gpu(a, b, c, d, solvedim)
    finally:
        O.set_option("trid_warp", -1)
    ref = d.copy()
    oracle_solve(orc, a, b, c, ref, solvedim)
    np.testing.assert_allclose(x, ref, rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("n", [300, 1000, 4099])
def test_long_strided_lines(gpu_runtime, orc, n):
    """y lines of any length (Thomas per line, scratch sized by the call)."""
    a, b, c, d = seeded.trid_system((n, 33), 1, n)
    x, _ = run_gpu(a, b, c, d, 1, pad=(0, 3))
    ref = d.copy()
    oracle_solve(orc, a, b, c, ref, 1)
    np.testing.assert_allclose(x, ref, rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_uneven_batch_one_launch(gpu_runtime, orc, solvedim):
    """Blocks of different edge sizes solved in a single persistent launch."""
    import torch
    rng_sizes = [(7, 19, 33), (32, 40, 50), (61, 5, 12), (13, 64, 100), (2, 3, 4), (40, 40, 40)]
    systems, host, dev = [], [], []
    for i, shp in enumerate(rng_sizes):
        a, b, c, d = seeded.trid_system(shp, solvedim, 100 + i)
        t = [torch.from_numpy(v).cuda() for v in (a, b, c, d)]
        dev.append(t)
        host.append((a, b, c, d))
        systems.append(dict(a=t[0].data_ptr(), b=t[1].data_ptr(), c=t[2].data_ptr(), d=t[3].data_ptr(), u=None,
                            dims=list(reversed(shp)), pads=list(reversed(shp))))
    O.reset_counters()
    O.trid_batch(8, solvedim, systems, None)
    torch.cuda.synchronize()
    assert O.counters()["kernels"] == 1
    for (a, b, c, d), t in zip(host, dev):
        ref = d.copy()
        oracle_solve(orc, a, b, c, ref, solvedim)
        np.testing.assert_allclose(t[3].cpu().numpy(), ref, rtol=1e-12, atol=1e-13)


def test_dat_api_with_range(gpu_runtime, orc):
    """ops_tridMultiDimBatch on dats over a sub-range (offset from the range
    as ops_tridiag.cpp:109-119 computes it), then _Inc along z."""
    nx, ny, nz = 20, 18, 16
    blk = O.ops_decl_block(3, "adi")
    a, b, c, d = seeded.trid_system((nz, ny, nx), 1, 7)
    mk = lambda v, name: O.ops_decl_dat(blk, 1, [nx, ny, nz], [0, 0, 0], [-1, -1, -1], [1, 1, 1],
                                       np.pad(v, 1), "double", name)
    da, db, dc, dd = mk(a, "a"), mk(b, "b"), mk(c, "c"), mk(d, "d")
    rng = [2, 15, 1, 17, 3, 12]
    O.ops_tridMultiDimBatch(3, 1, rng, da, db, dc, dd)
    got = O.ops_dat_fetch_data(dd)[1:-1, 1:-1, 1:-1]
    sub = (slice(rng[4], rng[5]), slice(rng[2], rng[3]), slice(rng[0], rng[1]))
    ref = d.copy()
    ra, rb, rc, rd = (np.ascontiguousarray(t[sub]) for t in (a, b, c, ref))
    oracle_solve(orc, ra, rb, rc, rd, 1)
    expect = d.copy()
    expect[sub] = rd
    np.testing.assert_allclose(got, expect, rtol=1e-12, atol=1e-13)
    u = mk(np.zeros_like(d), "u")
    O.ops_tridMultiDimBatch_Inc(3, 2, [0, nx, 0, ny, 0, nz], da, db, dc, dd, u)
    gu = O.ops_dat_fetch_data(u)[1:-1, 1:-1, 1:-1]
    ref2 = got.copy()
    oracle_solve(orc, a, b, c, ref2, 2)
    np.testing.assert_allclose(gu, ref2, rtol=1e-11, atol=1e-12)


def test_full_size_256_cube_residual(gpu_runtime):
    """Config-3 single block: 256^3 FP64, each direction; ||Ax - d||_inf / ||d||_inf."""
    import torch
    n = 256
    for solvedim in (0, 1, 2):
        a, b, c, d = seeded.trid_system((n, n, n), solvedim, 3 + solvedim)
        x, _ = run_gpu(a, b, c, d, solvedim)
        ax = 2 - solvedim
        xm = np.moveaxis(x, ax, -1)
        am, bm, cm, dm = (np.moveaxis(t, ax, -1) for t in (a, b, c, d))
        r = bm * xm - dm
        r[..., 1:] += am[..., 1:] * xm[..., :-1]
        r[..., :-1] += cm[..., :-1] * xm[..., 1:]
        assert np.abs(r).max() / np.abs(dm).max() < 1e-14
