"""ops_halo_transfer on the B200 vs the reference library (golden dumps of
oracle/ref_drivers/halo_cases.cpp) bit for bit, and vs the numpy oracle
(oracle/halo.py) on 3D, multi-component and mixed-precision cases."""
import os

import numpy as np
import pytest

from halo_cases import CASES, DM, DP, SIZE, initial, refill
from oracle import halo as ref
from ops_b200 import ops as O
from ops_b200._lib import OpsError

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "halo_cases.npz")


def test_matches_reference_cases(gpu_runtime):
    g = np.load(GOLDEN)
    g0 = O.ops_decl_block(2, "g0")
    g1 = O.ops_decl_block(2, "g1")
    host = initial()
    dats = {}
    for name, blk, t in (("a", g0, "double"), ("b", g1, "double"), ("bf", g1, "float")):
        dats[name] = O.ops_decl_dat(blk, 1, [SIZE, SIZE], [0, 0], [DM, DM], [DP, DP], host[name], t, name)
    for c, halos in enumerate(CASES):
        refill(host)
        for name, d in dats.items():
            O.ops_dat_set_data(d, host[name])
        hs = [O.ops_decl_halo(dats[s], dats[t], it, fb, tb, fd, td) for s, t, it, fb, tb, fd, td in halos]
        O.ops_halo_transfer(O.ops_decl_halo_group(hs))
        for name, d in dats.items():
            host[name] = O.ops_dat_fetch_data(d)
            assert np.array_equal(host[name], g[f"case{c}_{name}"]), (c, name)


def test_3d_permutations_components_and_conversion(gpu_runtime):
    rng = np.random.default_rng(11)
    b0 = O.ops_decl_block(3, "p")
    b1 = O.ops_decl_block(3, "q")
    size, dm, dp = [12, 9, 7], [-1, -2, -1], [2, 1, 2]
    ext = [s - m + p for s, m, p in zip(size, dm, dp)]
    arrays, dats, meta = {}, {}, {}
    for name, blk, t, dim, base in (("p", b0, "double", 2, [0, 0, 0]), ("q", b1, "double", 2, [3, -1, 2]),
                                    ("qf", b1, "float", 2, [0, 0, 0])):
        shp = tuple(reversed(ext)) + (dim,)
        arr = rng.standard_normal(shp).astype(np.float64 if t == "double" else np.float32)
        arrays[name] = arr
        dats[name] = O.ops_decl_dat(blk, dim, size, base, dm, dp, arr, t, name)
        meta[name] = (base, dm)
    # iteration box 3 x 4 x 5; target directions permute and flip the axes
    halos = [("p", "q", [3, 4, 5], [-1, 0, 2], [4, 0, 3], [1, 2, 3], [-3, 1, -2]),
             ("p", "qf", [5, 3, 4], [2, -2, 0], [0, 1, 2], [2, 3, -1], [1, -2, 3])]
    hs = [O.ops_decl_halo(dats[s], dats[t], it, fb, tb, fd, td) for s, t, it, fb, tb, fd, td in halos]
    O.ops_halo_transfer(O.ops_decl_halo_group(hs))
    ref.transfer(arrays, meta, halos)
    for name, d in dats.items():
        assert np.array_equal(O.ops_dat_fetch_data(d), arrays[name]), name


def test_rejects_boxes_outside_the_allocation(gpu_runtime):
    blk = O.ops_decl_block(2, "r")
    a = O.ops_decl_dat(blk, 1, [8, 8], [0, 0], [-1, -1], [1, 1], None, "double", "ra")
    b = O.ops_decl_dat(blk, 1, [8, 8], [0, 0], [-1, -1], [1, 1], None, "double", "rb")
    with pytest.raises(OpsError):
        O.ops_decl_halo(a, b, [2, 8], [8, 0], [-1, 0], [1, 2], [1, 2])   # source x 8..9: the ring ends at 8
    with pytest.raises(OpsError):
        O.ops_decl_halo(a, b, [2, 8], [0, 0], [0, 0], [1, 1], [1, 2])    # not a permutation
    ok = O.ops_decl_halo(a, b, [2, 8], [7, 0], [-1, 0], [1, 2], [1, 2])   # x 7..8 is inside
    assert ok >= 0
