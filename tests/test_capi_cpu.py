"""The C-ABI library loads and exports every declared symbol (no GPU calls)."""
import ctypes
import glob
import os
import re

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
