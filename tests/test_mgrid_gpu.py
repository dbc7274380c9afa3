"""Multigrid restrict/prolong stencils through the public API: the reference's
own mgrid test app (apps/c/mgrid/mgrid.cpp:54-260, zero-based variant)
restated with ops_b200.ops calls. Its two checks (prolong_check,
restrict_check) are the app's known answer: both flags must come back 0.
The fields are also compared with their closed forms, and a kernel without
`mgrid` must refuse a restrict stencil."""
import numpy as np
import pytest

from ops_b200 import ops as O
from ops_b200._lib import OpsError

pytestmark = pytest.mark.gpu


def run_mgrid_app():
    grid0 = O.ops_decl_block(2, "grid0")
    s00 = O.ops_decl_stencil(2, 1, [0, 0], "00")
    s5 = O.ops_decl_stencil(2, 5, [0, 0, -1, 0, 1, 0, 0, -1, 0, 1], "5pt")
    stride1 = [2, 2]
    prolong3 = O.ops_decl_prolong_stencil(2, 3, [0, 0, -1, 0, 1, 0], stride1, "PROLONG_00_M10_P10")
    restrict3 = O.ops_decl_restrict_stencil(2, 3, [0, 0, -1, 0, 1, 0], stride1, "RESTRICT_00_M10_P10")
    d_m, d_p, base = [-2, -2], [2, 2], [0, 0]
    size4, size0, size1 = [24, 24], [12, 12], [6, 6]
    data0 = O.ops_decl_dat(grid0, 1, size0, base, d_m, d_p, None, "double", "data0", stride=[2, 2])
    data1 = O.ops_decl_dat(grid0, 1, size1, base, d_m, d_p, None, "double", "data1", stride=[4, 4])
    data5 = O.ops_decl_dat(grid0, 1, size4, base, d_m, d_p, None, "double", "data5", stride=[1, 1])
    data6 = O.ops_decl_dat(grid0, 1, size0, base, d_m, d_p, None, "double", "data6", stride=[2, 2])
    data3 = O.ops_decl_dat(grid0, 1, size1, base, d_m, d_p, None, "double", "data3", stride=[4, 4])
    err = O.ops_decl_reduction_handle(4, "int", "reduct_err")

    d = [1, 2]
    groups = []
    # periodic halos in x and y for data5, in x for data0 and data1 (mgrid.cpp:120-172)
    h1 = O.ops_decl_halo(data5, data5, [2, size4[1] + 4], [0, -2], [size4[0], -2], d, d)
    h2 = O.ops_decl_halo(data5, data5, [2, size4[1] + 4], [size4[0] - 2, -2], [-2, -2], d, d)
    groups.append(O.ops_decl_halo_group([h1, h2]))
    h1 = O.ops_decl_halo(data5, data5, [size4[0] + 4, 2], [-2, 0], [-2, size4[1]], d, d)
    h2 = O.ops_decl_halo(data5, data5, [size4[0] + 4, 2], [-2, size4[1] - 2], [-2, -2], d, d)
    groups.append(O.ops_decl_halo_group([h1, h2]))
    h3 = O.ops_decl_halo(data0, data0, [2, size0[1] + 4], [0, -2], [size0[1], -2], d, d)
    h4 = O.ops_decl_halo(data0, data0, [2, size0[1] + 4], [size0[0] - 2, -2], [-2, -2], d, d)
    groups.append(O.ops_decl_halo_group([h3, h4]))
    h5 = O.ops_decl_halo(data1, data1, [2, size1[1] + 4], [0, -2], [size1[1], -2], d, d)
    h6 = O.ops_decl_halo(data1, data1, [2, size1[1] + 4], [size1[0] - 2, -2], [-2, -2], d, d)
    groups.append(O.ops_decl_halo_group([h5, h6]))

    r12, r24, r6 = [0, 12, 0, 12], [0, 24, 0, 24], [0, 6, 0, 6]
    O.ops_par_loop("mgrid/mgrid_populate_kernel_1", "mgrid_populate_kernel_1", grid0, 2, r6,
                   O.ops_arg_dat(data1, 1, s00, "double", O.OPS_WRITE), O.ops_arg_idx())
    O.ops_halo_transfer(groups[3])
    O.ops_par_loop("mgrid/mgrid_prolong_kernel", "mgrid_prolong_kernel", grid0, 2, r12,
                   O.ops_arg_dat(data1, 1, prolong3, "double", O.OPS_READ),
                   O.ops_arg_dat(data0, 1, s00, "double", O.OPS_WRITE), O.ops_arg_idx())
    O.ops_halo_transfer(groups[2])
    O.ops_par_loop("mgrid/mgrid_prolong_kernel", "mgrid_prolong_kernel", grid0, 2, r24,
                   O.ops_arg_dat(data0, 1, prolong3, "double", O.OPS_READ),
                   O.ops_arg_dat(data5, 1, s00, "double", O.OPS_WRITE), O.ops_arg_idx())
    O.ops_halo_transfer(groups[0])
    O.ops_halo_transfer(groups[1])
    O.ops_par_loop("mgrid/prolong_check", "prolong_check", grid0, 2, r24,
                   O.ops_arg_dat(data5, 1, s5, "double", O.OPS_READ), O.ops_arg_idx(),
                   O.ops_arg_reduce(err, 1, "int", O.OPS_MAX),
                   O.ops_arg_gbl(size4[0], 1, "int", O.OPS_READ), O.ops_arg_gbl(size4[1], 1, "int", O.OPS_READ))
    err_prolong = int(O.ops_reduction_result(err))
    prolonged = O.ops_dat_fetch_data(data5)

    O.ops_par_loop("mgrid/mgrid_populate_kernel_3", "mgrid_populate_kernel_3", grid0, 2, r24,
                   O.ops_arg_dat(data5, 1, s00, "double", O.OPS_WRITE), O.ops_arg_idx())
    O.ops_par_loop("mgrid/mgrid_restrict_kernel", "mgrid_restrict_kernel", grid0, 2, r12,
                   O.ops_arg_dat(data5, 1, restrict3, "double", O.OPS_READ),
                   O.ops_arg_dat(data6, 1, s00, "double", O.OPS_WRITE), O.ops_arg_idx())
    O.ops_par_loop("mgrid/mgrid_restrict_kernel", "mgrid_restrict_kernel", grid0, 2, r6,
                   O.ops_arg_dat(data6, 1, restrict3, "double", O.OPS_READ),
                   O.ops_arg_dat(data3, 1, s00, "double", O.OPS_WRITE), O.ops_arg_idx())
    O.ops_par_loop("mgrid/restrict_check", "restrict_check", grid0, 2, r6,
                   O.ops_arg_dat(data3, 1, s00, "double", O.OPS_READ), O.ops_arg_idx(),
                   O.ops_arg_reduce(err, 1, "int", O.OPS_MAX), O.ops_arg_gbl(size4[0], 1, "int", O.OPS_READ))
    err_restrict = int(O.ops_reduction_result(err))
    return err_prolong, err_restrict, prolonged, O.ops_dat_fetch_data(data6), O.ops_dat_fetch_data(data3), (
        data1, s00, grid0)


def interior(a, n, halo=2):
    return a[halo:halo + n, halo:halo + n]


def test_mgrid_app_checks_and_fields(gpu_runtime):
    ep, er, d5, d6, d3, _ = run_mgrid_app()
    assert ep == 0 and er == 0          # the app's own PASSED condition (mgrid.cpp:255)
    y, x = np.mgrid[0:24, 0:24]
    np.testing.assert_array_equal(interior(d5, 24), (x // 4 + (y // 4) * 6).astype(np.float64))
    y, x = np.mgrid[0:12, 0:12]
    np.testing.assert_array_equal(interior(d6, 12), (2 * x + 2 * y * 24).astype(np.float64))
    y, x = np.mgrid[0:6, 0:6]
    np.testing.assert_array_equal(interior(d3, 6), (4 * x + 4 * y * 24).astype(np.float64))


def test_plain_kernel_refuses_multigrid_stencil(gpu_runtime):
    *_, (data1, s00, grid0) = run_mgrid_app()
    r = O.ops_decl_restrict_stencil(2, 1, [0, 0], [2, 2], "R00")
    with pytest.raises(OpsError):
        O.ops_par_loop("mgrid/mgrid_populate_kernel_1", "bad", grid0, 2, [0, 3, 0, 3],
                       O.ops_arg_dat(data1, 1, r, "double", O.OPS_WRITE), O.ops_arg_idx())


def test_restrict_out_of_allocation_is_refused(gpu_runtime):
    *_, (data1, s00, grid0) = run_mgrid_app()
    fine = O.ops_decl_dat(grid0, 1, [8, 8], [0, 0], [-1, -1], [1, 1], None, "double", "fine8")
    coarse = O.ops_decl_dat(grid0, 1, [8, 8], [0, 0], [0, 0], [0, 0], None, "double", "coarse8")
    r = O.ops_decl_restrict_stencil(2, 1, [0, 0], [2, 2], "R00b")
    with pytest.raises(OpsError):       # 2 * 7 = 14 lies beyond the fine dat's 9
        O.ops_par_loop("mgrid/mgrid_restrict_kernel", "too far", grid0, 2, [0, 8, 0, 8],
                       O.ops_arg_dat(fine, 1, r, "double", O.OPS_READ),
                       O.ops_arg_dat(coarse, 1, s00, "double", O.OPS_WRITE), O.ops_arg_idx())
