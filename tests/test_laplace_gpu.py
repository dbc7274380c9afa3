"""Laplace Jacobi on the B200 path vs the oracle and the reference's golden
vectors: bit-exact fields and per-iteration max|delta| (integer-free FP64
work with identical operation order; the bar is equality)."""
import glob
import os

import numpy as np
import pytest

from ops_b200 import apps, seeded
from ops_b200 import ops as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu


def oracle_run(orc, field, iters):
    A = np.ascontiguousarray(field.copy())
    errs = np.zeros(max(iters, 1))
    orc.oracle_laplace_run(A.shape[1] - 2, A.shape[0] - 2, iters, A.ctypes.data, errs.ctypes.data)
    return A, errs[:iters]


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "laplace_seeded_*.npz"))))
def test_app_matches_reference_golden(gpu_runtime, path):
    g = np.load(path)
    init = seeded.laplace_field(int(g["imax"]), int(g["jmax"]), int(g["seed"]))
    A, errs, _ = apps.laplace2d(init, int(g["iters"]))
    assert np.array_equal(A, g["field"])
    assert np.array_equal(errs, g["errors"])


@pytest.mark.parametrize("imax,jmax,iters,seed", [
    (1, 1, 3, 2), (2, 1, 4, 3), (1, 9, 5, 4), (129, 3, 6, 5), (1000, 17, 7, 6), (300, 300, 20, 7),
    (4097, 5, 3, 8), (127, 255, 11, 9)])
def test_app_matches_oracle_edge_shapes(gpu_runtime, orc, imax, jmax, iters, seed):
    init = seeded.laplace_field(imax, jmax, seed)
    A, errs, _ = apps.laplace2d(init, iters)
    Ao, eo = oracle_run(orc, init, iters)
    assert np.array_equal(A, Ao)
    assert np.array_equal(errs, eo)


def test_app_full_size_matches_oracle(gpu_runtime, orc):
    """Config-1 grid (4096^2), a few iterations, bit-exact."""
    init = seeded.laplace_field(4096, 4096, 1)
    A, errs, _ = apps.laplace2d(init, 4)
    Ao, eo = oracle_run(orc, init, 4)
    assert np.array_equal(errs, eo)
    assert np.array_equal(A, Ao)


def test_step7_known_answer(gpu_runtime, orc):
    """apps/c/laplace2d_tutorial/step7: 4094^2, 100 iterations, sine boundary
    -> 2.421354960840227e-03 (reference tolerance 0.001 %); bit-exact vs the
    oracle on the same host-computed boundary."""
    init = np.zeros((4096, 4096))
    orc.oracle_laplace_step7_init(4094, 4094, init.ctypes.data)
    A, errs, _ = apps.laplace2d(init, 100)
    assert abs(errs[-1] / 2.421354960840227e-03 - 1.0) < 1e-5
    _, eo = oracle_run(orc, init, 100)
    assert np.array_equal(errs, eo)


def _api_run(field, iters, graphs, fusion):
    """The reference driver's loop sequence through the Python OPS mirror."""
    O.set_option("graphs", graphs)
    O.set_option("fusion", fusion)
    jmax, imax = field.shape[0] - 2, field.shape[1] - 2
    blk = O.ops_decl_block(2, "my_grid")
    A = O.ops_decl_dat(blk, 1, [imax, jmax], [0, 0], [-1, -1], [1, 1], None, "double", "A")
    An = O.ops_decl_dat(blk, 1, [imax, jmax], [0, 0], [-1, -1], [1, 1], None, "double", "Anew")
    S0 = O.ops_decl_stencil(2, 1, [0, 0], "0,0")
    S5 = O.ops_decl_stencil(2, 5, [0, 0, 1, 0, -1, 0, 0, 1, 0, -1], "5pt")
    h = O.ops_decl_reduction_handle(8, "double", "error")
    full = [-1, imax + 1, -1, jmax + 1]
    O.ops_par_loop("laplace2d/set_zero", "set zero", blk, 2, full, O.ops_arg_dat(A, 1, S0, "double", O.OPS_WRITE))
    O.ops_par_loop("laplace2d/set_zero", "set zero", blk, 2, full, O.ops_arg_dat(An, 1, S0, "double", O.OPS_WRITE))
    O.ops_dat_set_data(A, field)
    O.ops_dat_set_data(An, field)
    errs = []
    inner = [0, imax, 0, jmax]
    for _ in range(iters):
        O.ops_par_loop("laplace2d/apply_stencil", "apply stencil", blk, 2, inner,
                       O.ops_arg_dat(A, 1, S5, "double", O.OPS_READ),
                       O.ops_arg_dat(An, 1, S0, "double", O.OPS_WRITE),
                       O.ops_arg_reduce(h, 1, "double", O.OPS_MAX))
        errs.append(O.ops_reduction_result(h))
        O.ops_par_loop("laplace2d/copy", "copy", blk, 2, inner,
                       O.ops_arg_dat(A, 1, S0, "double", O.OPS_WRITE),
                       O.ops_arg_dat(An, 1, S0, "double", O.OPS_READ))
    out = O.ops_dat_fetch_data(A)
    O.set_option("graphs", 1)
    O.set_option("fusion", 1)
    return out, np.array(errs)


@pytest.mark.parametrize("graphs,fusion", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_python_api_path_matches_oracle(gpu_runtime, orc, graphs, fusion):
    init = seeded.laplace_field(211, 97, 13)
    A, errs = _api_run(init, 12, graphs, fusion)
    Ao, eo = oracle_run(orc, init, 12)
    assert np.array_equal(A, Ao)
    assert np.array_equal(errs, eo)


def test_copy_elision_and_graphs_are_used(gpu_runtime):
    init = seeded.laplace_field(256, 256, 3)
    O.reset_counters()
    apps.laplace2d(init, 10)
    c = O.counters()
    assert c["loops"] == 20
    assert c["graphs"] >= 1          # repeated flushes replay as CUDA graphs
    assert 0 < c["kernels"] <= 20    # copies became storage swaps


def test_errors_are_reported(gpu_runtime):
    blk = O.ops_decl_block(2, "g")
    A = O.ops_decl_dat(blk, 1, [8, 8], [0, 0], [-1, -1], [1, 1], None, "double", "A")
    S5 = O.ops_decl_stencil(2, 5, [0, 0, 1, 0, -1, 0, 0, 1, 0, -1], "5pt")
    with pytest.raises(O.OpsError):       # wrong arg count for the kernel
        O.ops_par_loop("laplace2d/apply_stencil", "x", blk, 2, [0, 8, 0, 8], O.ops_arg_dat(A, 1, S5, "double", 0))
    with pytest.raises(O.OpsError):       # unknown kernel
        O.ops_par_loop("laplace2d/nope", "x", blk, 2, [0, 8, 0, 8], O.ops_arg_dat(A, 1, S5, "double", 0))
    with pytest.raises(O.OpsError):       # wrong buffer size
        O.ops_dat_set_data(A, np.zeros(3))
    ptr, stride = O.ops_dat_get_raw_pointer(A, O.OPS_DEVICE)
    assert ptr and stride[0] >= 10
    with pytest.raises(O.OpsError):       # loop on a dat whose raw pointer is held
        O.ops_par_loop("laplace2d/set_zero", "z", blk, 2, [0, 8, 0, 8],
                       O.ops_arg_dat(A, 1, O.ops_decl_stencil(2, 1, [0, 0], "0"), "double", 1))
    O.ops_dat_release_raw_data(A, O.OPS_READ)
