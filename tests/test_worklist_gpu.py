"""Runs of one loop kernel over several blocks of different shapes (a
multi-block application's step over its blocks, e.g. apps/c/mblock) launched
as one kernel over a work list of their uneven domains (exec_loop_list):
the same values as one launch per loop, one launch for the run, and loops
that depend on one another kept apart."""
import numpy as np
import pytest

from ops_b200 import ops as O

pytestmark = pytest.mark.gpu
SHAPES = [(37, 23), (200, 5), (64, 64), (3, 300), (129, 17)]


def _setup():
    s00 = O.ops_decl_stencil(2, 1, [0, 0], "00")
    blocks, a, b = [], [], []
    for i, (nx, ny) in enumerate(SHAPES):
        blk = O.ops_decl_block(2, f"wl{i}")
        blocks.append(blk)
        a.append(O.ops_decl_dat(blk, 1, [nx, ny], [0, 0], [-1, -1], [1, 1], None, "double", f"wl_a{i}"))
        b.append(O.ops_decl_dat(blk, 1, [nx, ny], [0, 0], [-1, -1], [1, 1], None, "double", f"wl_b{i}"))
    return s00, blocks, a, b


def _run(lists):
    O.set_option("lists", lists)
    O.set_option("graphs", 0)
    s00, blocks, a, b = _setup()
    O.ops_execute()
    O.reset_counters()
    for i, (nx, ny) in enumerate(SHAPES):
        O.ops_par_loop("mgrid/mgrid_populate_kernel_1", "populate", blocks[i], 2, [0, nx, 0, ny],
                       O.ops_arg_dat(a[i], 1, s00, "double", O.OPS_WRITE), O.ops_arg_idx())
    O.ops_execute()
    k_populate = O.counters()["kernels"]
    O.reset_counters()
    for i, (nx, ny) in enumerate(SHAPES):
        O.ops_par_loop("laplace2d/copy", "copy", blocks[i], 2, [0, nx, 0, ny],
                       O.ops_arg_dat(b[i], 1, s00, "double", O.OPS_WRITE), O.ops_arg_dat(a[i], 1, s00, "double", O.OPS_READ))
    O.ops_execute()
    k_copy = O.counters()["kernels"]
    out = [(O.ops_dat_fetch_data(a[i]), O.ops_dat_fetch_data(b[i])) for i in range(len(SHAPES))]
    O.set_option("lists", 1)
    O.set_option("graphs", 1)
    return k_populate, k_copy, out


def test_uneven_blocks_in_one_launch(gpu_runtime):
    k_pop, k_copy, got = _run(1)
    assert (k_pop, k_copy) == (1, 1)
    k_pop1, k_copy1, ref = _run(0)
    assert (k_pop1, k_copy1) == (len(SHAPES), len(SHAPES))
    for i, (nx, ny) in enumerate(SHAPES):
        A, B = got[i]
        exp = np.zeros((ny + 2, nx + 2))
        y, x = np.mgrid[0:ny, 0:nx]
        exp[1:-1, 1:-1] = x + 6.0 * y
        assert np.array_equal(A, exp), i
        assert np.array_equal(B, exp), i
        assert np.array_equal(A, ref[i][0]) and np.array_equal(B, ref[i][1])


def test_dependent_loops_are_not_batched(gpu_runtime):
    """copy b <- a then c <- b on one block: the second reads what the first
    writes, so they launch separately (and c equals a)."""
    O.set_option("graphs", 0)
    s00 = O.ops_decl_stencil(2, 1, [0, 0], "00")
    blk = O.ops_decl_block(2, "dep")
    n = 48
    init = np.arange((n + 2) * (n + 2), dtype=np.float64).reshape(n + 2, n + 2)
    a = O.ops_decl_dat(blk, 1, [n, n], [0, 0], [-1, -1], [1, 1], init, "double", "dep_a")
    b = O.ops_decl_dat(blk, 1, [n, n], [0, 0], [-1, -1], [1, 1], None, "double", "dep_b")
    c = O.ops_decl_dat(blk, 1, [n, n], [0, 0], [-1, -1], [1, 1], None, "double", "dep_c")
    O.ops_execute()
    O.reset_counters()
    O.ops_par_loop("laplace2d/copy", "copy", blk, 2, [0, n, 0, n], O.ops_arg_dat(b, 1, s00, "double", O.OPS_WRITE),
                   O.ops_arg_dat(a, 1, s00, "double", O.OPS_READ))
    O.ops_par_loop("laplace2d/copy", "copy", blk, 2, [0, n, 0, n], O.ops_arg_dat(c, 1, s00, "double", O.OPS_WRITE),
                   O.ops_arg_dat(b, 1, s00, "double", O.OPS_READ))
    O.ops_execute()
    assert O.counters()["kernels"] == 2
    C = O.ops_dat_fetch_data(c)
    assert np.array_equal(C[1:-1, 1:-1], init[1:-1, 1:-1])
    O.set_option("graphs", 1)
