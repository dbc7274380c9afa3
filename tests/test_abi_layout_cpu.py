"""The ctypes mirrors in ops_b200/_lib.py have the layout of the C structs in
include/ops_b200.h: a small C program compiled here prints sizeof and every
member's offsetof, which must equal the ctypes figures."""
import ctypes
import os
import subprocess

import pytest

from ops_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PAIRS = [("ops_b200_arg", _lib.Arg), ("ops_b200_trid_system", _lib.TridSystem),
         ("ops_b200_kernel_stat", _lib.KernelStat), ("ops_b200_clover_state", _lib.CloverState),
         ("ops_b200_clover_deck", _lib.CloverDeck), ("ops_b200_clover3d_state", _lib.Clover3DState),
         ("ops_b200_clover3d_deck", _lib.Clover3DDeck), ("ops_b200_tea_deck", _lib.TeaDeck),
         ("ops_b200_heat_system", _lib.HeatSystem), ("ops_b200_heat_stats", _lib.HeatStats),
         ("ops_b200_heat_system3d", _lib.HeatSystem3D),
         ("ops_b200_heat_batch", _lib.HeatBatch), ("ops_b200_tridsolver_params", _lib.TridsolverParams)]


def c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ops_b200.h"', 'int main(void) {']
    for cname, cls in PAIRS:
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field in cls._fields_:
            lines.append(f'  printf("{cname} {field[0]} %zu\\n", offsetof({cname}, {field[0]}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {tuple(l.split()[:2]): int(l.split()[2]) for l in out.splitlines()}


@pytest.fixture(scope="module")
def layout(tmp_path_factory):
    return c_layout(tmp_path_factory.mktemp("abi"))


@pytest.mark.parametrize("cname,cls", PAIRS, ids=[p[0] for p in PAIRS])
def test_struct_layout(layout, cname, cls):
    assert layout[(cname, "sizeof")] == ctypes.sizeof(cls)
    for field in cls._fields_:
        assert layout[(cname, field[0])] == getattr(cls, field[0]).offset, field[0]
