"""The C-ABI library loads and exports every declared symbol (no GPU calls)."""
import ctypes
import glob
import os
import re

import pytest

import ops_b200.build as build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(ops_b200_\w+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_builds_and_exports_all_declared_symbols():
    path = build.build()
    L = ctypes.CDLL(path)
    missing = [n for n in sorted(_declared()) if not hasattr(L, n)]
    assert not missing, missing
    assert len(_declared()) >= 20


def test_init_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        return
    from ops_b200 import ops
    from ops_b200._lib import OpsError
    try:
        ops.ops_init(0, 0)
    except OpsError as e:
        assert e.code == -2 and "no CUDA device" in str(e)
    else:
        raise AssertionError("ops_init succeeded without a GPU")


def test_calls_before_init_are_rejected():
    from ops_b200 import lib
    L = lib()
    assert L.ops_b200_decl_block(2, b"x") == -3
    assert b"ops_b200_init" in L.ops_b200_last_error()
    assert L.ops_b200_has_kernel(b"laplace2d/apply_stencil") == 1
    assert L.ops_b200_has_kernel(b"nope/none") == 0


def test_single_process_api_calls_without_gpu(capsys):
    """ops_printf / ops_fprintf / ops_partition / ops_tridsolver_params need
    no device: printing, a no-op partition, setters that steer nothing."""
    import io

    from ops_b200 import ops as O
    O.ops_printf("%d cells, %s\n", 42, "ok")
    assert capsys.readouterr().out == "42 cells, ok\n"
    s = io.StringIO()
    O.ops_fprintf(s, "x=%.2f\n", 1.5)
    assert s.getvalue() == "x=1.50\n"
    assert O.ops_partition("") is None
    p = O.ops_tridsolver_params(None, O.ops_tridsolver_params.PCR)
    p.set_jacobi_params(1e-10, 1e-12, 5)
    p.set_batch_size(64)
    p.set_cuda_opts(1, 2, 3)
    p.set_cuda_sync(0)
    assert (p.strategy, p.jacobi, p.batch_size, p.cuda_opts, p.cuda_sync) == (3, (1e-10, 1e-12, 5), 64, (1, 2, 3), 0)
    # the C-ABI struct holds the same values
    c = p._p
    assert (c.strategy, c.jacobi_rtol, c.jacobi_atol, c.jacobi_maxiter, c.batch_size, list(c.cuda_opts),
            c.cuda_sync) == (3, 1e-10, 1e-12, 5, 64, [1, 2, 3], 0)
    assert O.ops_tridsolver_params(None)._p.strategy == O.ops_tridsolver_params.GATHER_SCATTER
    with pytest.raises(O.OpsError):
        O.ops_tridsolver_params(None, 9)
    with pytest.raises(O.OpsError):
        p.set_batch_size(-1)


def test_heat_solve_arguments_are_checked_before_any_device_work():
    """Unknown methods, bad shapes and bad tolerances are refused with
    OPS_B200_ERR_ARG before the library touches a GPU (the field pointers
    below are never dereferenced)."""
    import ctypes as C

    from ops_b200 import lib
    from ops_b200._lib import HeatStats, HeatSystem
    L = lib()
    fake = C.c_void_p(4096)
    sysd = HeatSystem(64, 64, 66, fake, fake, fake, fake, 1.0, 1.0)
    st = HeatStats()
    assert L.ops_b200_heat_solve(C.byref(sysd), 7, -1, 1e-10, 100, 0, None, C.byref(st), None) == -1
    assert b"method" in L.ops_b200_last_error()
    assert L.ops_b200_heat_solve(C.byref(sysd), 5, -1, 0.0, 100, 0, None, C.byref(st), None) == -1
    bad = HeatSystem(64, 64, 65, fake, fake, fake, fake, 1.0, 1.0)      # pitch < nx + 2
    assert L.ops_b200_heat_solve(C.byref(bad), 5, -1, 1e-10, 100, 0, None, C.byref(st), None) == -1
    assert L.ops_b200_heat_mg_apply(C.byref(bad), fake, fake, None, None) == -1
    assert b"shape" in L.ops_b200_last_error()


def test_heat_solve3d_arguments_are_checked_before_any_device_work():
    """The 3D solve refuses a plane other than pitch * (ny + 2), a pitch
    below nx + 2, methods other than the two PCG rules, a non-positive
    tolerance and null fields with OPS_B200_ERR_ARG, before any device work."""
    import ctypes as C

    from ops_b200 import lib
    from ops_b200._lib import HeatStats, HeatSystem3D
    L = lib()
    fake = C.c_void_p(4096)
    st = HeatStats()

    def solve(nx, ny, nz, pitch, plane, method=1, eps=1e-10, ptr=fake):
        sysd = HeatSystem3D(nx, ny, nz, pitch, plane, ptr, fake, fake, fake, fake, 1.0, 1.0, 1.0)
        return L.ops_b200_heat_solve3d(C.byref(sysd), method, eps, 100, C.byref(st), None)

    assert solve(8, 8, 8, 10, 99) == -1                  # plane != pitch * (ny + 2)
    assert b"shape" in L.ops_b200_last_error()
    assert solve(8, 8, 8, 9, 90) == -1                   # pitch < nx + 2
    assert solve(8, 8, 0, 10, 100) == -1                 # empty
    assert solve(8, 8, 8, 10, 100, method=3) == -1       # the learned FCG is 2D only (methods 0, 1, 2)
    assert b"method" in L.ops_b200_last_error()
    assert solve(8, 8, 8, 10, 100, eps=0.0) == -1
    assert solve(8, 8, 8, 10, 100, ptr=None) == -1       # null Kx
    assert b"null" in L.ops_b200_last_error()
