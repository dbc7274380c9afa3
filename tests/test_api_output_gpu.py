"""Output, timing and host-data calls of the reference's single-process API
(ops_timing_output, ops_diagnostic_output, ops_print_dat_to_txtfile,
ops_get_data / ops_put_data) through the Python mirror, on Laplace loops."""
import io

import numpy as np
import pytest

from ops_b200 import ops as O

pytestmark = pytest.mark.gpu


def laplace_setup(name, nx=20, ny=12):
    blk = O.ops_decl_block(2, name)
    A = O.ops_decl_dat(blk, 1, [nx, ny], [0, 0], [-1, -1], [1, 1], None, "double", name + "_A")
    An = O.ops_decl_dat(blk, 1, [nx, ny], [0, 0], [-1, -1], [1, 1], None, "double", name + "_Anew")
    S0 = O.ops_decl_stencil(2, 1, [0, 0], name + "_0")
    S5 = O.ops_decl_stencil(2, 5, [0, 0, 1, 0, -1, 0, 0, 1, 0, -1], name + "_5")
    h = O.ops_decl_reduction_handle(8, "double", name + "_err")
    field = np.random.default_rng(3).uniform(0, 1, (ny + 2, nx + 2))
    O.ops_dat_set_data(A, field)
    O.ops_dat_set_data(An, np.zeros_like(field))
    return blk, A, An, S0, S5, h, field


def sweep(blk, A, An, S0, S5, h, nx=20, ny=12):
    O.ops_par_loop("laplace2d/apply_stencil", "apply stencil", blk, 2, [0, nx, 0, ny],
                   O.ops_arg_dat(A, 1, S5, "double", O.OPS_READ), O.ops_arg_dat(An, 1, S0, "double", O.OPS_WRITE),
                   O.ops_arg_reduce(h, 1, "double", O.OPS_MAX))
    return O.ops_reduction_result(h)


def test_timing_and_diagnostic_output(gpu_runtime, capsys):
    O.ops_init(0, 3)
    try:
        blk, A, An, S0, S5, h, _ = laplace_setup("outgrid")
        O.clear_kernel_timing()
        for _ in range(3):
            sweep(blk, A, An, S0, S5, h)
        out = io.StringIO()
        O.ops_timing_output(out)
        text = out.getvalue()
        assert "Count Time     MPI-time     Bandwidth(GB/s)" in text
        row = [l for l in text.splitlines() if l.startswith("laplace2d/apply_stencil")]
        assert row and row[0].split()[1] == "3"
        assert "Total kernel time:" in text
        O.ops_diagnostic_output()
        diag = capsys.readouterr().out
        assert "OPS diagnostic output" in diag and "outgrid" in diag
        assert "outgrid_A" in diag and "[22][14]" in diag and "[-1][-1]" in diag
    finally:
        O.ops_init(0, 0)
    out = io.StringIO()
    O.ops_timing_output(out)                 # diags <= 1: nothing, as in the reference
    assert out.getvalue() == ""


def test_print_dat_and_host_data(gpu_runtime, tmp_path):
    blk, A, An, S0, S5, h, field = laplace_setup("dumpgrid")
    f = tmp_path / "dump.txt"
    O.ops_print_dat_to_txtfile(A, str(f))
    lines = f.read_text().splitlines()
    assert lines[0].strip() == "ops_dat:  dumpgrid_A"
    assert lines[2].startswith("block Dims : 2 [22][14]")
    assert lines[3].strip() == "elem size 8"
    vals = np.array([[float(v) for v in l.split()] for l in lines[4:]])
    np.testing.assert_allclose(vals, field, atol=1e-10)
    sweep(blk, A, An, S0, S5, h)
    got = O.ops_get_data(An)
    want = np.zeros_like(field)
    want[1:-1, 1:-1] = 0.25 * (field[1:-1, 2:] + field[1:-1, :-2] + field[:-2, 1:-1] + field[2:, 1:-1])
    np.testing.assert_array_equal(got[1:-1, 1:-1], want[1:-1, 1:-1])
    O.ops_put_data(An, field * 2)
    np.testing.assert_array_equal(O.ops_dat_fetch_data(An), field * 2)
